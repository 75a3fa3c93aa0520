"""Splits a .curc archive into its payloads (reference layout:
preprocess.cpp:261-276 archive header, compress.cu:1364-2146 block body,
read back by decompress.cu:760-814)."""
import struct


def split_archive(data: bytes):
    po, pe, L, nblocks = struct.unpack_from("<BBHB", data, 0)
    off = 5
    blocks = []
    for _ in range(nblocks):
        b = {}
        b["reads_count"], = struct.unpack_from("<I", data, off); off += 4
        b["decoder_table"] = data[off:off + 16]; off += 16
        if po:
            b["join_std"] = data[off]; off += 1
        b["ref_std"] = data[off]; off += 1
        b["sizes"] = struct.unpack_from("<QQQ", data, off); off += 24
        names = []
        if po:
            names.append("id_pos")
        names += ["strand", "ref"]
        if not po:
            names += ["read_off", "unmap_n_read_off", "unmap_read_off"]
            if pe:
                names.append("pe_order")
        names += ["ref_off_map", "ref_len_map", "unmap_ref_off_map", "unmap_ref_len_map", "unmap_n_ref_off_map",
                  "unmap_n_ref_len_map", "mismatch_count", "mismatch_base"]
        for nm in names:
            n, = struct.unpack_from("<Q", data, off); off += 8
            b[nm] = data[off:off + n]; off += n
        mm = data[off]; off += 1
        b["max_mismatch"] = mm
        for m in range(1, mm + 1):
            n, = struct.unpack_from("<Q", data, off); off += 8
            b[f"mis_off_{m}"] = data[off:off + n]; off += n
        blocks.append(b)
    assert off == len(data), (off, len(data))
    return {"preserve_order": po, "paired_end": pe, "read_len": L, "blocks": blocks}

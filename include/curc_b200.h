/* C-ABI of the B200 pseudogenome path of CURC.
 *
 * Plain pointers and sizes only.  Every function returns 0 on success and a
 * negative code on failure; curc_last_error() gives the message.  A context
 * owns one CUDA stream and a device arena on one GPU; it is not thread safe
 * (use one context per thread).  Device pointers passed in must be on the
 * context's device; `stream` arguments are cudaStream_t values (NULL = the
 * context's own stream).
 *
 * The reference has no library boundary: its seam is two C++ functions,
 *   encode(char* buffer, const Param&, size_t n, size_t start, uint64_t* reads_db_host, size_t W)
 *       src/compress.cuh:56, src/compress.cu:2151-2180
 *   block_compress(uint64_t* reads_db_host, vector<uint32_t> reads_id, vector<char> N_reads_db_host,
 *                  vector<uint32_t> N_reads_id, const Param&, uint8_t block_id, int device_count)
 *       src/compress.cuh:48, src/compress.cu:1349-2148
 * and the `curc -c` command line (src/main.cpp:53-161).  The entry points
 * below replace those, one for one where noted.
 */
#ifndef CURC_B200_H
#define CURC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct curc_ctx curc_ctx;

#define CURC_OK 0
#define CURC_ERR_ARG (-1)
#define CURC_ERR_CUDA (-2)
#define CURC_ERR_STATE (-3)
#define CURC_ERR_IO (-4)

/* Creates a context on `device` (get_device_count_and_init,
 * src/compress.cu:2183-2195, per device). */
int curc_ctx_create(int device, curc_ctx** out);
/* The same, returning at once: the CUDA set-up (driver start, context, the
 * pipeline's stream; about a second on a fresh process) runs on a thread of
 * its own.  curc_compress_files parses its FASTQ input meanwhile; every
 * other call waits for the set-up and returns its error, if it failed.
 * curc_ctx_wait waits for it explicitly.  No reference counterpart. */
int curc_ctx_create_deferred(int device, curc_ctx** out);
int curc_ctx_wait(curc_ctx* ctx);
void curc_ctx_destroy(curc_ctx* ctx);
/* Last error message of the context (or of creation when ctx is NULL). */
const char* curc_last_error(const curc_ctx* ctx);

/* 2-bit packing of n reads of length L held as n*L ASCII bytes on the
 * device; writes n*ceil(L/32) packed words and one N flag per read (1 when
 * the read contains 'N').  Replaces encode(), src/compress.cu:2151-2180,
 * plus the N test of src/preprocess.cpp:149-152. */
int curc_pack_device(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, uint64_t* packed_dev,
                     uint8_t* has_n_dev, void* stream);

/* Same packing, plus the N split of src/preprocess.cpp:147-193 (ids of the
 * reads without N and of those with N, each ascending; counts_dev[0] and
 * counts_dev[1] receive their numbers), without allocating device memory:
 * for callers that manage all device memory through their own pool or that
 * cannot take the device synchronisation a cudaMalloc may cause.  No
 * counterpart in the reference.  Its scratch is a fixed array of about 512
 * KB inside the library (held on every GPU that loads it until exit), which
 * limits a call to 2^27 reads; larger calls return CURC_ERR_ARG.  Calls share
 * that array, so calls that overlap on the GPU race; stream-ordered calls do
 * not.  The first call on a device sets up the array's address and should
 * come before any stream capture; that address is kept for the process and
 * is not valid after cudaDeviceReset on the device.  No context: errors are
 * read with curc_last_error(NULL). */
int curc_pack_split_noalloc(int device, const char* seqs_dev, uint64_t n, uint16_t read_len, uint64_t* packed_dev,
                            uint8_t* has_n_dev, uint32_t* reads_id_dev, uint32_t* n_reads_id_dev,
                            uint32_t* counts_dev, void* stream);

/* Compresses one block.  `seqs` holds n reads of length read_len as ASCII
 * (host memory), in block order (paired end: mates interleaved, as
 * src/preprocess.cpp:147-193 numbers them).  Runs the whole device path
 * (pack, sort/dedupe, k-mer index, overlap linking, chain filter, full
 * match, assembly, mapping, stream emission, unmapped pseudogenomes,
 * reverse-complement repeat removal) and keeps every stream in the context
 * until the next call.  Replaces block_compress(), src/compress.cu:1349-2148
 * up to (not including) the entropy coders. */
int curc_block_run(curc_ctx* ctx, const char* seqs, uint64_t n, uint16_t read_len, int preserve_order,
                   int paired_end);

/* Same with the reads already on the device (n*read_len bytes). */
int curc_block_run_device(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, int preserve_order,
                          int paired_end);

/* Whether block runs also copy the stage intermediates ("packed",
 * "sorted_ids", "next", "prev", "offset", "ref_ids", "unmatch_ids", "hq_seq",
 * "hq_records", "map_*") to the host for parity checks (default 1).  The
 * streams are always returned.  No reference counterpart. */
int curc_ctx_keep_intermediates(curc_ctx* ctx, int keep);

/* Frees the device memory a context keeps between blocks: its pipeline's
 * arena and the extra pipelines, input slots and pinned staging of the
 * batched path (they are made again on the next run or drain).  Results of
 * the last run stay readable.  CURC_ERR_STATE while blocks are queued.  No
 * reference counterpart. */
int curc_ctx_trim(curc_ctx* ctx);

/* Autotuner (no counterpart in the reference).  Knobs, in this order: the
 * overlap index's bucket table size as a multiple of the prefix count
 * {1, 2, 4, 8}, presence-bitmap bits per prefix {8, 16, 32}, overlap passes
 * between host reads of the link count {2, 4, 8, 16}, threads per block of
 * the mapping kernel {64, 128, 256}, and the form of the full-match pass
 * loop: a launch per kernel from the host (0), one CUDA graph whose
 * conditional while node replays the passes (1), or one persistent
 * cooperative kernel that runs every pass (2).  None changes any result: every stream
 * is the same under every setting; only the time does.  curc_autotune runs
 * the given block (device memory) under the candidates one knob at a time,
 * keeps the fastest, and sets it on the context; with cache_path, choices
 * are read from and saved to that file per (read length, read count rounded
 * down to a power of two), and *from_cache tells whether the file had one.
 * The k-mer length and the other derived parameters are part of the format
 * and are not tuned. */
int curc_ctx_set_tuning(curc_ctx* ctx, const int32_t* knobs); /* knobs[5] */
int curc_ctx_get_tuning(curc_ctx* ctx, int32_t* knobs);       /* knobs[5] */
int curc_autotune(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, int preserve_order,
                  int paired_end, const char* cache_path, int* from_cache);
/* Loads a cache file written by curc_autotune: every later block run of the
 * context (batched blocks included) uses the choice of its own (read
 * length, read-count bucket), or the context's setting when the bucket has
 * none.  NULL or "" stops using it. */
int curc_ctx_use_tuning_cache(curc_ctx* ctx, const char* cache_path);

/* Learned mode of whole-file compression (no counterpart in the reference;
 * the plain coders are the reference's, src/compress.cu:1923-2146).  With a
 * model set (the bytes curc_learn_model returns), curc_compress_files also
 * codes each block's mismatch bases and offsets with the learned coder and
 * keeps, per block, the smaller of the two codings; a learned block marks
 * its mismatch-base container with the coder byte 100 (the reference's
 * decoder cannot read such blocks, the product decoder can).  NULL or 0
 * bytes restores plain mode, whose archives are the reference's byte for
 * byte.  CURC_ERR_ARG when the size is not a model's. */
int curc_ctx_set_mismatch_model(curc_ctx* ctx, const void* model, uint64_t bytes);

/* Whole-file compression, the drop-in for `curc -c` (src/main.cpp:53-161,
 * src/preprocess.cpp:66-283 and the coders of src/compress.cu:1923-2146):
 * reads f1 (and f2 for paired end, else NULL) with the reference's block
 * split, runs each block through the device path, codes its streams with
 * the reference's coders (fast-lzma2 at `flzma2_level` with
 * `flzma2_threads`, PPMd7/LZMA, CLR range coder, and the `bsc` executable at
 * bsc_path, which writes scratch files in tmpdir) and writes the archive to
 * archive_path in the reference's .curc layout.  Coding of a block overlaps
 * the next block's ingest and device work.  *reads_out / *blocks_out (may be
 * NULL) receive the totals. */
int curc_compress_files(curc_ctx* ctx, const char* f1, const char* f2, const char* archive_path, double block_ratio,
                        int preserve_order, int flzma2_level, int flzma2_threads, const char* bsc_path,
                        const char* tmpdir, uint64_t* reads_out, uint32_t* blocks_out);

/* One block's streams to its archive body in the reference's block layout
 * (compress.cu:1364-2146), host only: the coders curc_compress_files uses,
 * on streams named as curc_block_get names them ("decoder_table", "sizes",
 * "strand", "ref", "unmap_ref", "unmap_n_ref", "id_to_pos" or "read_off",
 * "unmap_read_off", "unmap_n_read_off", "pe_order", the six repeat maps,
 * "mis_cnt", "mis_base", "mis_off_<m>"), e.g. those a curc_batch_drain
 * callback reads.  count streams: names[i], ptrs[i], sizes[i] bytes.  The
 * strand stream goes through the `bsc` executable at bsc_path (scratch files
 * in tmpdir).  *out (free it with curc_buffer_free) receives the body,
 * *out_bytes its size; a missing stream gives CURC_ERR_STATE. */
int curc_encode_block(uint32_t reads_count, uint16_t read_len, int preserve_order, int paired_end,
                      const char* const* names, const void* const* ptrs, const uint64_t* sizes, uint32_t count,
                      int flzma2_level, int flzma2_threads, const char* bsc_path, const char* tmpdir, char** out,
                      uint64_t* out_bytes);
void curc_buffer_free(char* p);
/* The 5-byte archive header (preprocess.cpp:261-266) into out5: an archive
 * is this header followed by its block bodies in order (at most 254). */
int curc_archive_header(int preserve_order, int paired_end, uint16_t read_len, uint32_t blocks, char* out5);

/* FASTQ ingest alone, host only (the block split of process(),
 * preprocess.cpp:66-254): reads f1 (and f2 for paired end, else NULL) in
 * the reference's windows, cuts blocks where it does, and calls
 * block(user, index, seqs, n, read_len) once per block with its n reads
 * (n x read_len ASCII bytes in block order, mates interleaved; valid during
 * the call), e.g. to queue them with curc_batch_submit after a copy.  A
 * non-zero return from block stops with CURC_ERR_STATE; unreadable or
 * malformed input gives CURC_ERR_IO.  *reads_out / *blocks_out (may be
 * NULL) receive the totals. */
typedef int (*curc_fastq_block_fn)(void* user, uint32_t index, const char* seqs, uint64_t n, uint16_t read_len);
int curc_fastq_blocks(const char* f1, const char* f2, double block_ratio, curc_fastq_block_fn block, void* user,
                      uint64_t* reads_out, uint32_t* blocks_out);

/* Layout of a .curc archive without decoding it, host only: its flags,
 * read length, block count, and per block its body size in bytes and its
 * read count (block_bytes / block_reads hold up to 254 entries; any output
 * pointer may be NULL). */
int curc_archive_info(const char* archive_path, int* preserve_order, int* paired_end, uint16_t* read_len,
                      uint32_t* blocks, uint64_t* block_bytes, uint32_t* block_reads);

/* Number of CUDA devices (the reference CLI's "GPU device count" line,
 * compress.cu:2183-2190). */
int curc_device_count(int* count);

/* Whole-archive decompression, the drop-in for `curc -d` (src/decompress.cu:
 * 760-1060, src/decompress.cpp): reads the .curc archive at archive_path and
 * writes <out_prefix>.seq (single end) or <out_prefix>_1.seq and
 * <out_prefix>_2.seq (paired end), one read per line, byte for byte what the
 * reference decoder writes.  Host only: needs no context and no GPU.  The
 * strand stream goes through the `bsc` executable at bsc_path, with scratch
 * files in tmpdir; threads = host threads (0: all).  *reads_out (may be
 * NULL) receives the read count.  Errors (CURC_ERR_IO for files,
 * CURC_ERR_STATE for a malformed archive) are described by
 * curc_last_error(NULL). */
int curc_decompress_file(const char* archive_path, const char* out_prefix, const char* bsc_path, const char* tmpdir,
                         int threads, uint64_t* reads_out);

/* Host view of a named result of the last block run ("strand", "mis_cnt",
 * "mis_base", "read_off", "ref", ... and the stage intermediates
 * "sorted_ids", "next", "prev", "offset", "hq_seq", ...).  The pointer stays
 * valid until the next run or destroy.  Returns CURC_ERR_ARG for an unknown
 * name. */
int curc_block_get(curc_ctx* ctx, const char* name, const void** ptr, uint64_t* bytes);

/* Batched path: blocks queued on a context and run by several block
 * pipelines at once (the context's own and curc_batch_workers - 1 more, each
 * with its own stream and device memory), so that one block's copies and
 * host round trips overlap another's kernels.  Replaces the reference's
 * one-thread-per-block scheduling of process() (preprocess.cpp:195-242) and
 * its GPU mutexes (compress.cu:52-65) on one device.
 *
 * curc_batch_submit queues n x read_len ASCII reads (host memory that must
 * stay valid until the drain returns) and returns a ticket.  curc_batch_drain
 * runs every queued block (blocks of at least 2^28 bases first, double-buffered
 * from the calling thread; the rest on concurrent pipelines); after each one it
 * calls done(user, ticket) (one call at a time, in completion order, from the
 * thread that ran the block),
 * during which curc_block_get on that thread returns that block's results.
 * A non-zero return from done stops the drain with CURC_ERR_STATE.
 * curc_batch_workers sets the number of pipelines (1..16, default 2). */
typedef int (*curc_block_done_fn)(void* user, uint32_t ticket);
int curc_batch_submit(curc_ctx* ctx, const char* seqs, uint64_t n, uint16_t read_len, int preserve_order,
                      int paired_end, uint32_t* ticket);
int curc_batch_workers(curc_ctx* ctx, int workers);
int curc_batch_drain(curc_ctx* ctx, curc_block_done_fn done, void* user);

/* Learned coder of the mismatch streams (no counterpart in the reference,
 * whose plain method codes bases and counts with PPMd7, compress.cu:1931-1933,
 * and offsets with the CLR range coder, util.cuh:307-343).  A small network
 * (int8 weights, int32 accumulation, integer frequencies) predicts, walking
 * each read with mismatches, the gap to the next mismatch and the read's base
 * there from the surrounding pseudogenome; a range coder uses its 12-bit
 * frequencies.  Training (FP32 forward, backward and Adam on the GPU) uses the
 * anchors of blocks added with curc_learn_add_block; curc_learn_train also
 * quantises.  curc_learn_encode codes the mismatch gaps and bases of the
 * context's last block; curc_learn_decode_check decodes a stream on the host
 * and compares it with that block (*ok = 1 when lossless). */
typedef struct curc_learn curc_learn;
int curc_learn_create(int device, curc_learn** out);
void curc_learn_destroy(curc_learn* l);
const char* curc_learn_error(const curc_learn* l);
int curc_learn_add_block(curc_learn* l, curc_ctx* ctx);
uint64_t curc_learn_anchors(const curc_learn* l);
int curc_learn_train(curc_learn* l, int epochs, int batch, float lr, uint64_t seed, float* final_loss);
int curc_learn_model(curc_learn* l, const void** ptr, uint64_t* bytes);
int curc_learn_set_model(curc_learn* l, const void* ptr, uint64_t bytes);
int curc_learn_encode(curc_learn* l, curc_ctx* ctx, const void** out, uint64_t* bytes);
int curc_learn_decode_check(curc_learn* l, curc_ctx* ctx, const void* data, uint64_t bytes, int* ok);
/* Test support: runs the tensor-core inference over the context's last
 * block and recomputes each anchor's frequencies with the host integer
 * model; *mismatched counts anchors whose frequencies differ. */
int curc_learn_infer_check(curc_learn* l, curc_ctx* ctx, uint64_t* anchors, uint64_t* mismatched);
/* Test support: loss and gradients of one FP32 forward/backward pass over n
 * dense inputs (n x 128) with base / gap targets (-1: none), for the parameter
 * vector `params` (curc_learn_param_count floats: W1 128x128, b1, W2 128x128,
 * b2, W3 20x128, b3). */
uint64_t curc_learn_param_count(void);
int curc_learn_grad(curc_learn* l, const float* params, const float* x, const int8_t* tb, const int8_t* tg,
                    uint32_t n, float* loss, float* grads);
/* Coded sizes, with the reference's plain coders, of the context's last
 * block's mismatch streams: out[0] counts, out[1] bases, out[2] offsets. */
int curc_plain_mismatch_bytes(curc_ctx* ctx, uint64_t* out);
/* Bytes of the same mismatch streams of the context's last block (counts,
 * bases, offsets; each coded on its own) under fast-lzma2 level 10 (out[0])
 * and libbsc through the bsc executable (out[1]), for comparison with the
 * learned coder.  No counterpart in the reference. */
int curc_mismatch_general_bytes(curc_ctx* ctx, const char* bsc_path, const char* tmpdir, uint64_t* out);

/* Number of kernels the library has launched in this process (no
 * reference counterpart; used to report launches per benchmark step). */
uint64_t curc_kernel_launches(void);

/* Milliseconds of device time of the last block run, by stage
 * (CUDA events on the context's stream): "pack", "sort_dedupe", "overlap",
 * "chain_filter", "full_match", "assembly", "mapping", "emit",
 * "unmapped_refs", "refmatch", and "total" (the whole run).  After
 * curc_compress_files, also its host-stage wall times summed over blocks:
 * "files.total", "files.ingest", "files.device", "files.snapshot",
 * "files.coders" (coder threads), "files.until_last_block",
 * "files.coder_tail" (coding left after the last block ran), and
 * "coder.<stream>" per coder ("id_pos", "strand", "ref", "maps",
 * "mis_cnt", "mis_base", "mis_off", "read_off", "pe_order"). */
int curc_block_stage_ms(curc_ctx* ctx, const char* stage, float* ms);

#ifdef __cplusplus
}
#endif

#endif

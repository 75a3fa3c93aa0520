// `curc` command line on the B200 path (options of src/main.cpp:55-67).
// Compression: `curc -c -i in.fastq[,in_2.fastq] -o name [--working_dir d]
// [--block_ratio r] [--flzma2_level l] [--flzma2_thread_num t]
// [--preserve_order]` writes <working_dir>/<name>.curc.
// Decompression: `curc -d -i in.curc -o name [--working_dir d]` writes
// <working_dir>/<name>.seq (or <name>_1.seq and <name>_2.seq), host only.
#include <thread>
#include <dlfcn.h>
#include <limits.h>
#include <stdlib.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/curc_b200.h"

namespace {

bool has_ext(const std::string& p, const char* a, const char* b = nullptr) {
    auto ends = [&](const char* e) {
        const size_t n = std::strlen(e);
        return p.size() >= n && p.compare(p.size() - n, n, e) == 0;
    };
    return ends(a) || (b && ends(b));
}

std::string self_dir() {
    char buf[PATH_MAX];
    const ssize_t k = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    if (k <= 0) return ".";
    buf[k] = 0;
    std::string s(buf);
    return s.substr(0, s.find_last_of('/'));
}

int usage() {
    std::puts(
        "curc (B200 path)\n"
        "  -c, --compress            compress file\n"
        "  -d, --decompress          decompress archive\n"
        "  -i, --input arg           input path (paired-end fastq paths are separated by commas)\n"
        "  -o, --output arg          output file name\n"
        "      --working_dir arg     working directory (default .)\n"
        "      --block_ratio arg     ratio of block size (default 1)\n"
        "      --flzma2_level arg    fast-lzma2 compression level [1...10] (default 10)\n"
        "      --flzma2_thread_num   fast-lzma2 thread number (default 16)\n"
        "      --preserve_order      preserve order information\n"
        "      --device arg          CUDA device (default 0)\n"
        "      --coder arg           mismatch coder: plain (the reference's streams, default) or learned\n"
        "                            (per block, the learned coder where it is smaller; needs --model)\n"
        "      --model arg           learned mismatch model file (from the training API)\n"
        "  -v, --version             print version\n"
        "  -h, --help                print usage\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    bool comp = false, decomp = false, po = false;
    std::string input, output, wd = ".";
    double ratio = 1.0;
    int level = 10, threads = 16, device = 0;
    std::string coder = "plain", model_path;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        try {
            if (a == "-c" || a == "--compress") comp = true;
            else if (a == "-d" || a == "--decompress") decomp = true;
            else if (a == "-i" || a == "--input") input = val();
            else if (a == "-o" || a == "--output") output = val();
            else if (a == "--working_dir") wd = val();
            else if (a == "--block_ratio") ratio = std::stod(val());
            else if (a == "--flzma2_level") level = std::stoi(val());
            else if (a == "--flzma2_thread_num") threads = std::stoi(val());
            else if (a == "--preserve_order") po = true;
            else if (a == "--device") device = std::stoi(val());
            else if (a == "--coder") coder = val();
            else if (a == "--model") model_path = val();
            else if (a == "-h" || a == "--help") return usage();
            else if (a == "-v" || a == "--version") {
                std::puts("v1.0.0");  // the archive format version (CURC 1.0.0)
                return 0;
            }
            else if (a == "--decode_buffer_size") val();
            else throw std::runtime_error("unknown option " + a);
        } catch (const std::exception& e) {
            std::printf("%s\n", e.what());
            return 0;
        }
    }
    if (input.empty() || output.empty() || (!comp && !decomp)) return usage();
    if (comp && decomp) {
        std::puts("compression and decompression options conflict");
        return 0;
    }
    struct stat st;
    if (stat(wd.c_str(), &st) != 0) {
        std::puts("invalid working dir");
        return 0;
    }
    if (decomp) {
        // src/main.cpp:139-152: one archive path ending in .curc
        if (input.find(',') != std::string::npos) {
            std::puts("invalid input path number");
            return 0;
        }
        if (stat(input.c_str(), &st) != 0 || !has_ext(input, ".curc")) {
            std::puts("please check the archive path (filename extension is .curc)");
            return 0;
        }
        std::string tmp = wd + "/curc_tmp_XXXXXX";
        if (!mkdtemp(&tmp[0])) {
            std::puts("cannot create a working directory");
            return 1;
        }
        uint64_t reads = 0;
        const int rc = curc_decompress_file(input.c_str(), (wd + "/" + output).c_str(), (self_dir() + "/bsc").c_str(),
                                            tmp.c_str(), 0, &reads);
        rmdir(tmp.c_str());
        if (rc != CURC_OK) {
            std::fprintf(stderr, "curc: %s\n", curc_last_error(nullptr));
            return 1;
        }
        return 0;  // the reference's decoder prints nothing either
    }
    if (!(ratio > 0 && ratio <= 1)) {
        std::puts("block ratio is a float number in the range (0,1]");
        return 0;
    }
    std::vector<std::string> files;
    size_t p = 0;
    while (p <= input.size()) {
        const size_t q = input.find(',', p);
        files.push_back(input.substr(p, q == std::string::npos ? std::string::npos : q - p));
        if (q == std::string::npos) break;
        p = q + 1;
    }
    if (files.empty() || files.size() > 2) {
        std::puts("invalid input path number");
        return 0;
    }
    for (size_t k = 0; k < files.size(); ++k) {
        if (stat(files[k].c_str(), &st) != 0 || !has_ext(files[k], ".fastq", ".fq")) {
            std::printf("please check the %s fastq path (filename extension is .fastq or .fq)\n",
                        k == 0 ? "first" : "second");
            return 0;
        }
    }
    std::string model;
    if (coder == "learned") {
        FILE* mf = model_path.empty() ? nullptr : std::fopen(model_path.c_str(), "rb");
        if (!mf) {
            std::puts("--coder learned needs a readable --model file");
            return 0;
        }
        char buf[1 << 16];
        size_t k;
        while ((k = std::fread(buf, 1, sizeof(buf), mf)) > 0) model.append(buf, k);
        std::fclose(mf);
    } else if (coder != "plain") {
        std::puts("--coder is plain or learned");
        return 0;
    }
    // the CUDA set-up runs on its own thread while the FASTQ input is read
    curc_ctx* ctx = nullptr;
    if (curc_ctx_create_deferred(device, &ctx) != CURC_OK) {
        std::fprintf(stderr, "GPU assert: %s\n", curc_last_error(nullptr));
        return 1;
    }
    if (!model.empty() && curc_ctx_set_mismatch_model(ctx, model.data(), model.size()) != CURC_OK) {
        std::printf("%s\n", curc_last_error(ctx));
        curc_ctx_destroy(ctx);
        return 0;
    }
    // the reference's progress lines (compress.cu:2183-2190, preprocess.cpp),
    // printed when the set-up has finished
    int init_rc = CURC_OK;
    std::thread announce([&] {
        init_rc = curc_ctx_wait(ctx);
        if (init_rc != CURC_OK) return;
        int devices = 0;
        curc_device_count(&devices);
        std::printf("gpu context init finish\n");
        std::printf("GPU device count : %d\n", devices);
        std::fflush(stdout);
    });
    std::string tmp = wd + "/curc_tmp_XXXXXX";
    if (!mkdtemp(&tmp[0])) {
        announce.join();
        std::puts("cannot create a working directory");
        return 1;
    }
    const std::string archive = wd + "/" + output + ".curc";
    const std::string bsc = self_dir() + "/bsc";
    uint64_t reads = 0;
    uint32_t blocks = 0;
    const int rc = curc_compress_files(ctx, files[0].c_str(), files.size() > 1 ? files[1].c_str() : nullptr,
                                       archive.c_str(), ratio, po, level, threads, bsc.c_str(), tmp.c_str(), &reads,
                                       &blocks);
    announce.join();
    rmdir(tmp.c_str());
    if (init_rc != CURC_OK) {
        std::fprintf(stderr, "GPU assert: %s\n", curc_last_error(ctx));
        return 1;
    }
    if (rc != CURC_OK) {
        std::fprintf(stderr, "curc: %s\n", curc_last_error(ctx));
        curc_ctx_destroy(ctx);
        return 1;
    }
    struct stat ast;
    stat(archive.c_str(), &ast);
    std::printf("reads count : %llu \n", (unsigned long long)reads);
    std::printf("block count : %u \n", blocks);
    std::printf("waiting block compress ...\n");
    std::vector<uint64_t> block_bytes(256, 0);
    uint32_t nb = 0;
    if (curc_archive_info(archive.c_str(), nullptr, nullptr, nullptr, &nb, block_bytes.data(), nullptr) == CURC_OK)
        for (uint32_t b = 0; b < nb; ++b)
            std::printf("block %u compress finish, compressed size : %llu\n", b, (unsigned long long)block_bytes[b]);
    std::printf("archive size : %lld bytes \n", (long long)ast.st_size);
    // the archive is closed: leave without tearing the CUDA context and its
    // device memory down one allocation at a time (the driver releases them
    // with the process)
    std::fflush(stdout);
    std::fflush(stderr);
    _exit(0);
}

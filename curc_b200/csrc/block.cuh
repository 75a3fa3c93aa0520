// Device-resident state of one block and the pipeline driver.
#pragma once
#include <map>
#include <string>
#include <vector>

#include "stages.cuh"

namespace curc {

// CUDA events around each stage on the block's stream.
struct StageTimer {
    cudaStream_t s;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> ev;
    void begin(const std::string& name) {
        cudaEvent_t a, b;
        CURC_CHECK(cudaEventCreate(&a));
        CURC_CHECK(cudaEventCreate(&b));
        CURC_CHECK(cudaEventRecord(a, s));
        ev.push_back({name, {a, b}});
    }
    void end() { CURC_CHECK(cudaEventRecord(ev.back().second.second, s)); }
    void collect(std::map<std::string, float>& out) {
        CURC_CHECK(cudaStreamSynchronize(s));
        for (auto& e : ev) {
            float ms = 0;
            CURC_CHECK(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
            out[e.first] += ms;
            cudaEventDestroy(e.second.first);
            cudaEventDestroy(e.second.second);
        }
        ev.clear();
    }
};

struct Block {
    cudaStream_t stream = nullptr;
    Arena arena;
    bool keep_intermediates = true;

    BlockParams p;
    uint32_t n = 0, m = 0, NN = 0, n_ref = 0, U = 0;
    uint64_t* db = nullptr;
    uint32_t *reads_id = nullptr, *n_ids = nullptr, *sorted = nullptr, *next = nullptr, *prev = nullptr;
    uint32_t *ref_ids = nullptr, *unmatch_ids = nullptr;
    uint16_t* offset = nullptr;
    uint8_t* nreads = nullptr;
    uint64_t* udb = nullptr;
    Assembled hq;
    MapOut mo;
    OverlapStats ostats;
    // emission
    uint32_t n_map = 0, n_records = 0, n_ug = 0, n_un = 0, n_mis = 0;
    uint32_t *ug = nullptr, *un = nullptr, *pe_order = nullptr;
    uint64_t* id_to_pos = nullptr;
    DevRecord* srec = nullptr;
    uint8_t *smis = nullptr, *mctx = nullptr, *mbase = nullptr;
    std::vector<uint32_t> class_count;
    uint64_t class_elems = 0;
    uint16_t* off_all = nullptr;
    Assembled lq, lqn;

    std::map<std::string, std::vector<uint8_t>> host;
    std::map<std::string, float> stage_ms;

    Block() { CURC_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
    ~Block() {
        if (stream) cudaStreamDestroy(stream);
    }
    Block(const Block&) = delete;
    Block& operator=(const Block&) = delete;

    void run(const uint8_t* d_seq, uint64_t n_reads, int L, bool po, bool pe);
    // a10-a12: stream emission, unmapped pseudogenomes, repeat removal
    void emit(StageTimer& T);
    // a12 on the three pseudogenomes; fills the ref / map streams
    void refmatch_all();

    template <class T>
    void keep(const std::string& name, const T* dev, size_t count) {
        auto& v = host[name];
        v.resize(count * sizeof(T));
        if (count) CURC_CHECK(cudaMemcpyAsync(v.data(), dev, count * sizeof(T), cudaMemcpyDeviceToHost, stream));
    }
};

}  // namespace curc

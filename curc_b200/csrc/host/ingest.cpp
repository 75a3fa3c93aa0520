// FASTQ ingest with the reference's block split (preprocess.cpp:66-254).
//
// The windows and block boundaries are the reference's; the files are mapped
// (as the reference maps them) and each window is parsed in place, its work
// spread over host threads: its newlines are counted per chunk, and every
// chunk then copies the sequence lines (line 1 of each 4-line record) it
// starts to their slots in the caller's buffer (mates interleaved).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>

#include "../../../include/curc_b200.h"
#include "host.hpp"

namespace curc {
namespace host {

namespace {

// Fixed team of threads running one indexed job at a time.  Tasks are
// claimed from a (generation, index) word by compare-and-swap, so a thread
// still finishing one job never claims a task of the next.
class Team {
public:
    explicit Team(int n) : size_(n) {
        for (int i = 1; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~Team() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    int size() const { return size_; }
    // Runs f(0..tasks-1) on the team and the caller; rethrows the first error.
    void run(int tasks, const std::function<void(int)>& f) {
        uint32_t g0;
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &f;
            tasks_ = tasks;
            left_ = tasks;
            err_ = nullptr;
            g0 = uint32_t(++gen_);
            claim_.store(uint64_t(g0) << 32);
        }
        cv_.notify_all();
        work(g0, &f, tasks);
        std::unique_lock<std::mutex> g(mu_);
        done_.wait(g, [&] { return left_ == 0; });
        job_ = nullptr;
        if (err_) std::rethrow_exception(err_);
    }

private:
    void work(uint32_t gen, const std::function<void(int)>* job, int tasks) {
        for (;;) {
            uint64_t v = claim_.load();
            int t;
            for (;;) {
                if (uint32_t(v >> 32) != gen || int(v & 0xFFFFFFFFu) >= tasks) return;
                if (claim_.compare_exchange_weak(v, v + 1)) break;
            }
            t = int(v & 0xFFFFFFFFu);
            try {
                (*job)(t);
            } catch (...) {
                std::lock_guard<std::mutex> g(mu_);
                if (!err_) err_ = std::current_exception();
            }
            std::lock_guard<std::mutex> g(mu_);
            if (--left_ == 0) done_.notify_all();
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            int tasks;
            uint32_t gen;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                if (!job_) continue;
                job = job_;
                tasks = tasks_;
                gen = uint32_t(gen_);
            }
            work(gen, job, tasks);
        }
    }
    int size_;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int tasks_ = 0, left_ = 0;
    std::atomic<uint64_t> claim_{0};
    uint64_t gen_ = 0;
    bool stop_ = false;
    std::exception_ptr err_;
};

struct File {
    int fd = -1;
    uint64_t size = 0;
    explicit File(const std::string& p) {
        fd = ::open(p.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("cannot open " + p);
        struct stat st;
        if (fstat(fd, &st) != 0) throw std::runtime_error("cannot stat " + p);
        size = uint64_t(st.st_size);
    }
    ~File() {
        if (map_ && map_ != MAP_FAILED) ::munmap(map_, size_t(size));
        if (fd >= 0) ::close(fd);
    }
    // the whole file, mapped read-only (the windows are parsed in place, with
    // no copy out of the page cache)
    const char* map() {
        if (!map_) {
            map_ = size ? ::mmap(nullptr, size_t(size), PROT_READ, MAP_PRIVATE, fd, 0) : nullptr;
            if (map_ == MAP_FAILED) throw std::runtime_error("cannot map the input file");
            if (map_) ::madvise(map_, size_t(size), MADV_SEQUENTIAL);
        }
        return static_cast<const char*>(map_);
    }
    void* map_ = nullptr;
    void read_range(uint64_t off, size_t n, char* dst) const {
        size_t got = 0;
        while (got < n) {
            const ssize_t k = ::pread(fd, dst + got, n - got, off_t(off + got));
            if (k <= 0) throw std::runtime_error("short read");
            got += size_t(k);
        }
    }
};

// Record-boundary heuristic of preprocess.cpp:114-137: scanning back from the
// window end, the cut is the first line start '@' whose bytes repeat, at the
// same columns, more than 5 consecutive bytes of the window's first line
// (the run counter carries over between candidates, as in the reference).
size_t cut_window(const char* b, size_t end) {
    if (b[0] != '@') throw std::runtime_error("io_buffer doesn't start with @");
    size_t fl = 0;
    while (fl < end && b[fl] != '\n') ++fl;
    if (fl == end) throw std::runtime_error("no record boundary found in a 50 MB window");
    size_t ne = end - fl;
    int eq = 0;
    while (ne > 0) {
        if (b[ne - 1] == '\n' && b[ne] == '@') {
            for (size_t j = 0; j < fl; ++j) {
                if (b[j] == b[ne + j]) {
                    if (++eq > 5) return ne;
                } else {
                    eq = 0;
                }
            }
        }
        --ne;
    }
    throw std::runtime_error("no record boundary found in a 50 MB window");
}

// Sequence lines of the records in b[0, end) (which starts at a record and
// ends after a newline) to dst + record * stride; returns the record count.
// Every sequence line must hold L bases (preprocess.cpp:147-160).
uint64_t parse_window(const char* b, size_t end, int L, char* dst, size_t stride, Team& team) {
    if (end == 0) return 0;
    if (b[end - 1] != '\n') throw std::runtime_error("truncated FASTQ record");
    const int T = std::max(1, std::min(team.size() * 4, int(end / 65536) + 1));
    const size_t piece = (end + T - 1) / T;
    std::vector<uint64_t> nl(T + 1, 0);
    team.run(T, [&](int t) {
        const size_t a = std::min(end, size_t(t) * piece), e = std::min(end, a + piece);
        nl[t + 1] = uint64_t(std::count(b + a, b + e, '\n'));
    });
    for (int t = 0; t < T; ++t) nl[t + 1] += nl[t];
    const uint64_t lines = nl[T];
    if (lines % 4) throw std::runtime_error("truncated FASTQ record");
    team.run(T, [&](int t) {
        const size_t a = std::min(end, size_t(t) * piece), e = std::min(end, a + piece);
        // lines starting in [a, e): at a (if a line starts there) and after
        // every newline before e - 1
        uint64_t li = nl[t];
        size_t p = a;
        if (a > 0 && b[a - 1] != '\n') {
            const char* q = static_cast<const char*>(std::memchr(b + a, '\n', e - a));
            if (!q) return;
            p = size_t(q - b) + 1;
            ++li;
        }
        while (p < e && p < end) {
            const char* q = static_cast<const char*>(std::memchr(b + p, '\n', end - p));
            const size_t le = size_t(q - b);
            if ((li & 3) == 1) {
                if (le - p != size_t(L)) throw std::runtime_error("read length isn't fix");
                std::memcpy(dst + (li >> 2) * stride, b + p, size_t(L));
            }
            ++li;
            p = le + 1;
        }
    });
    return lines / 4;
}

}  // namespace

int first_read_length(const std::string& f1) {
    File f(f1);
    std::vector<char> b(size_t(std::min<uint64_t>(f.size, 1 << 16)) + 1);
    f.read_range(0, b.size() - 1, b.data());
    b.back() = '\0';
    size_t e1 = 0;
    while (e1 + 1 < b.size() && b[e1] != '\n') ++e1;
    size_t e2 = e1 + 1;
    while (e2 + 1 < b.size() && b[e2] != '\n') ++e2;
    if (e2 + 1 >= b.size()) throw std::runtime_error("cannot read the first record of " + f1);
    return int(e2 - e1 - 1);
}

IngestResult ingest_fastq(const std::string& f1, const std::string& f2, double ratio, IngestSink& sink) {
    IngestResult res;
    const bool pe = !f2.empty();
    File a(f1);
    std::unique_ptr<File> b;
    if (pe) {
        b.reset(new File(f2));
        if (b->size != a.size) throw std::runtime_error("paired-end file size isn't equal");
    }
    const int L = first_read_length(f1);
    if (L < 1 || (L + 31) / 32 > 16) throw std::runtime_error("Read length must be less than 512");
    res.read_len = L;
    const uint64_t fq = a.size;
    const uint64_t block_bytes = pe ? uint64_t(2 * double(fq) * ratio) : uint64_t(double(fq) * ratio);
    const uint64_t win = pe ? 25000000 : 50000000;
    const int mates = pe ? 2 : 1;
    Team team(int(std::max(1u, std::min(32u, std::thread::hardware_concurrency()))));
    uint64_t total = 0, last_total = 0;
    const char* A = a.map();
    const char* B = pe ? b->map() : nullptr;
    bool open = false;
    auto begin_block = [&] {
        // sequence bytes of the block are at most its FASTQ bytes
        const uint64_t rest = (fq - total) * mates;
        sink.begin_block(size_t(std::min(rest, block_bytes + 2 * win * mates)), L);
        open = true;
    };
    while (total < fq) {
        if (!open) begin_block();
        size_t end = size_t(std::min(win, fq - total));
        const char* wa = A + total;
        const char* wb = pe ? B + total : nullptr;
        total += end;
        if (total < fq) {
            const size_t ne = cut_window(wa, end);
            total -= (end - ne);
            end = ne;
        }
        char* dst = sink.window_buffer(end * mates);
        const uint64_t n = parse_window(wa, end, L, dst, size_t(L) * mates, team);
        if (pe && parse_window(wb, end, L, dst + L, size_t(L) * mates, team) != n)
            throw std::runtime_error("paired-end files hold different record counts");
        sink.window_done(n * mates);
        res.reads += n * mates;
        uint64_t brb = total - last_total;
        if (pe) brb *= 2;
        if (brb > block_bytes) {
            sink.end_block();
            open = false;
            ++res.blocks;
            if (res.blocks >= 255) throw std::runtime_error("too many blocks");
            last_total = total;
        }
    }
    if (open) {
        sink.end_block();
        ++res.blocks;
        if (res.blocks >= 255) throw std::runtime_error("too many blocks");
    }
    return res;
}

}  // namespace host
}  // namespace curc

namespace curc {
std::string& ctxless_error();

namespace {
// Ingest sink that hands each block's reads, in host memory, to a callback.
class HostSink : public host::IngestSink {
public:
    HostSink(curc_fastq_block_fn fn, void* user) : fn_(fn), user_(user) {}
    void begin_block(size_t max_bytes, int L) override {
        L_ = L;
        off_ = 0;
        reserve(max_bytes);
    }
    char* window_buffer(size_t bytes) override {
        reserve(off_ + bytes);
        return buf_.get() + off_;
    }
    void window_done(uint64_t reads) override { off_ += size_t(reads) * size_t(L_); }
    void end_block() override {
        const uint64_t n = off_ / size_t(L_);
        if (fn_(user_, index_++, buf_.get(), n, uint16_t(L_)) != 0)
            throw std::logic_error("curc_fastq_blocks stopped by the callback");
    }

private:
    // grows keeping the bytes already written (no zero fill of new space)
    void reserve(size_t bytes) {
        if (bytes <= cap_) return;
        std::unique_ptr<char[]> nb(new char[bytes]);
        if (off_) std::memcpy(nb.get(), buf_.get(), off_);
        buf_ = std::move(nb);
        cap_ = bytes;
    }
    curc_fastq_block_fn fn_;
    void* user_;
    std::unique_ptr<char[]> buf_;
    size_t cap_ = 0;
    size_t off_ = 0;
    int L_ = 1;
    uint32_t index_ = 0;
};
}  // namespace
}  // namespace curc

extern "C" int curc_fastq_blocks(const char* f1, const char* f2, double block_ratio, curc_fastq_block_fn block,
                                 void* user, uint64_t* reads_out, uint32_t* blocks_out) {
    if (!f1 || !block) {
        curc::ctxless_error() = "curc_fastq_blocks: null path or callback";
        return CURC_ERR_ARG;
    }
    if (!(block_ratio > 0 && block_ratio <= 1)) {
        curc::ctxless_error() = "block ratio is a float number in the range (0,1]";
        return CURC_ERR_ARG;
    }
    try {
        curc::HostSink sink(block, user);
        const auto r = curc::host::ingest_fastq(f1, f2 ? f2 : "", block_ratio, sink);
        if (reads_out) *reads_out = r.reads;
        if (blocks_out) *blocks_out = uint32_t(r.blocks);
        return CURC_OK;
    } catch (const std::logic_error& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_STATE;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_IO;
    }
}

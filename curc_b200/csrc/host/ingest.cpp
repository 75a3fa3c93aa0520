// FASTQ ingest with the reference's block split (preprocess.cpp:66-254).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstring>
#include <memory>
#include <stdexcept>

#include "host.hpp"

namespace curc {
namespace host {

namespace {

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
        if (fd >= 0) ::close(fd);
    }
    void read_at(uint64_t off, size_t n, std::vector<char>& buf) const {
        buf.resize(n + 1);
        size_t got = 0;
        while (got < n) {
            const ssize_t k = ::pread(fd, buf.data() + got, n - got, off_t(off + got));
            if (k <= 0) throw std::runtime_error("short read");
            got += size_t(k);
        }
        buf[n] = '\0';
    }
};

// Record-boundary heuristic of preprocess.cpp:114-137: scanning back from the
// window end, the cut is the first line start '@' whose bytes repeat, at the
// same columns, more than 5 consecutive bytes of the window's first line
// (the run counter carries over between candidates, as in the reference).
size_t cut_window(const std::vector<char>& b, size_t end) {
    if (b[0] != '@') throw std::runtime_error("io_buffer doesn't start with @");
    size_t fl = 0;
    while (b[fl] != '\n') ++fl;
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

// One record's sequence line (preprocess.cpp:147-160); `lim` bounds the
// scan (a record cut off by the end of the data is an error).
inline const char* next_sequence(const std::vector<char>& b, size_t lim, size_t& i, int L) {
    auto line_end = [&](size_t k) {
        while (k < lim && b[k] != '\n') ++k;
        if (k >= lim) throw std::runtime_error("truncated FASTQ record");
        return k;
    };
    i = line_end(i) + 1;
    const size_t st = i;
    i = line_end(i);
    if (long(i - st) != L) throw std::runtime_error("read length isn't fix");
    i = line_end(i + 1) + 1;
    i = line_end(i) + 1;
    return b.data() + st;
}

}  // namespace

int first_read_length(const std::string& f1) {
    File f(f1);
    std::vector<char> b;
    f.read_at(0, size_t(std::min<uint64_t>(f.size, 1 << 16)), b);
    size_t e1 = 0;
    while (e1 < b.size() && b[e1] != '\n') ++e1;
    size_t e2 = e1 + 1;
    while (e2 < b.size() && b[e2] != '\n') ++e2;
    if (e2 >= b.size()) throw std::runtime_error("cannot read the first record of " + f1);
    return int(e2 - e1 - 1);
}

IngestResult ingest_fastq(const std::string& f1, const std::string& f2, double ratio,
                          const std::function<void(std::vector<char>&&, uint64_t, int)>& sink) {
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
    uint64_t total = 0, last_total = 0;
    std::vector<char> wa, wb, seqs;
    uint64_t n = 0;
    auto flush = [&] {
        sink(std::move(seqs), n, L);
        seqs = std::vector<char>();
        res.reads += n;
        n = 0;
        ++res.blocks;
        if (res.blocks >= 255) throw std::runtime_error("too many blocks");
    };
    while (total < fq) {
        size_t end = size_t(std::min(win, fq - total));
        a.read_at(total, end, wa);
        if (pe) b->read_at(total, end, wb);
        total += end;
        if (total < fq) {
            const size_t ne = cut_window(wa, end);
            total -= (end - ne);
            end = ne;
        }
        size_t i = 0, j = 0;
        const size_t lim_b = pe ? wb.size() - 1 : 0;
        while (i < end) {
            const char* s1 = next_sequence(wa, wa.size() - 1, i, L);
            seqs.insert(seqs.end(), s1, s1 + L);
            ++n;
            if (pe) {
                const char* s2 = next_sequence(wb, lim_b, j, L);
                seqs.insert(seqs.end(), s2, s2 + L);
                ++n;
            }
        }
        uint64_t brb = total - last_total;
        if (pe) brb *= 2;
        if (brb > block_bytes) {
            flush();
            last_total = total;
        }
    }
    if (total - last_total > 0) flush();
    return res;
}

}  // namespace host
}  // namespace curc

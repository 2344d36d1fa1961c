// nersc_host.cpp -- host side of NERSC configuration I/O (see nersc_host.h).
#include "nersc_host.h"

#include <errno.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/mag_c.h"

namespace magb {
namespace nersc {

namespace {

constexpr int kLineMax = 4096;

// snatch_keyword (field-matrix.h:575-592): 1 = found (value in v), 0 = not in
// this line, -1 = keyword without '='
int snatch(const char* line, const char* key, std::string& v) {
    if (!strstr(line, key)) return 0;
    const char* p = strchr(line, '=');
    if (!p) return -1;
    p++;
    while (*p == ' ' || *p == '\t') p++;
    v.assign(p);
    if (!v.empty() && v.back() == '\n') v.pop_back();
    return 1;
}

bool parse_hex32(const std::string& s, uint32_t& out) {
    const char* b = s.c_str();
    char* e = nullptr;
    const unsigned long long x = strtoull(b, &e, 16);
    if (e == b) return false;
    out = (uint32_t)x;  // stol(desc, 0, 16) assigned to a uint32_t
    return true;
}

// GF(2) 32x32 matrices: column i = image of register bit i
struct Gf2 {
    uint32_t c[32];
};
uint32_t apply(const Gf2& m, uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; v; i++, v >>= 1)
        if (v & 1u) r ^= m.c[i];
    return r;
}
Gf2 compose(const Gf2& a, const Gf2& b) {  // a after b
    Gf2 r;
    for (int i = 0; i < 32; i++) r.c[i] = apply(a, b.c[i]);
    return r;
}
Gf2 identity() {
    Gf2 r;
    for (int i = 0; i < 32; i++) r.c[i] = 1u << i;
    return r;
}
// advance of the register over n zero bytes
Gf2 zero_bytes(uint64_t n) {
    Gf2 bit;  // one zero bit: r -> (r >> 1) ^ (r & 1 ? poly : 0)
    bit.c[0] = 0xEDB88320u;
    for (int i = 1; i < 32; i++) bit.c[i] = 1u << (i - 1);
    Gf2 p = compose(bit, bit);
    p = compose(p, p);
    p = compose(p, p);  // one byte
    Gf2 r = identity();
    while (n) {
        if (n & 1) r = compose(p, r);
        p = compose(p, p);
        n >>= 1;
    }
    return r;
}
// the operator as four byte tables, so one application is four lookups
struct ByteTables {
    uint32_t t[4][256];
    explicit ByteTables(const Gf2& m) {
        for (int k = 0; k < 4; k++)
            for (int b = 0; b < 256; b++) t[k][b] = apply(m, (uint32_t)b << (8 * k));
    }
    uint32_t operator()(uint32_t v) const {
        return t[0][v & 0xffu] ^ t[1][(v >> 8) & 0xffu] ^ t[2][(v >> 16) & 0xffu] ^ t[3][v >> 24];
    }
};

}  // namespace

int read_header(FILE* f, Header& h, std::string& err) {
    h = Header();
    if (fseeko(f, 0, SEEK_SET) != 0) {
        err = "cannot rewind the file";
        return MAG_ERR_IO;
    }
    char line[kLineMax];
    std::string v;
    static const char* dim_keys[4] = {"DIMENSION_1", "DIMENSION_2", "DIMENSION_3", "DIMENSION_4"};
    while (fgets(line, sizeof(line), f)) {
        int r;
        if ((r = snatch(line, "DATATYPE", v)) != 0) {
            if (r < 0) { err = "DATATYPE line without '='"; return MAG_ERR_FORMAT; }
            h.datatype = v;
        }
        for (int d = 0; d < 4; d++)
            if ((r = snatch(line, dim_keys[d], v)) != 0) {
                if (r < 0) { err = std::string(dim_keys[d]) + " line without '='"; return MAG_ERR_FORMAT; }
                h.dims[d] = atoi(v.c_str());
            }
        if ((r = snatch(line, "CHECKSUM", v)) != 0) {
            if (r < 0 || !parse_hex32(v, h.checksum)) { err = "unreadable CHECKSUM"; return MAG_ERR_FORMAT; }
            h.has_checksum = true;
        }
        if ((r = snatch(line, "PLAQUETTE", v)) != 0) {
            if (r < 0) { err = "PLAQUETTE line without '='"; return MAG_ERR_FORMAT; }
            h.plaquette = strtod(v.c_str(), nullptr);
            h.has_plaquette = true;
        }
        if ((r = snatch(line, "LINK_TRACE", v)) > 0) {
            h.link_trace = strtod(v.c_str(), nullptr);
            h.has_link_trace = true;
        }
        if ((r = snatch(line, "CRC32HASH", v)) > 0) h.has_crc32 = parse_hex32(v, h.crc32);
        if (strstr(line, "END_HEADER")) {
            h.payload_offset = (long long)ftello(f);
            break;
        }
    }
    if (ferror(f)) {
        err = "read error in the header";
        return MAG_ERR_IO;
    }
    if (h.payload_offset < 0) {
        err = "no END_HEADER line";
        return MAG_ERR_FORMAT;
    }
    return MAG_OK;
}

int datatype_rows(const std::string& datatype, int& two_row, std::string& err) {
    if (datatype == "4D_SU3_GAUGE") two_row = 1;
    else if (datatype == "4D_SU3_GAUGE_3x3") two_row = 0;
    else {
        err = "WRONG DATATYPE '" + datatype + "'";
        return MAG_ERR_FORMAT;
    }
    return MAG_OK;
}

std::string format_header(const int dims[4], int two_row, uint32_t crc32, uint32_t checksum, double link_trace,
                          double plaquette, const char* ensemble_label, int sequence_number, double beta,
                          long long unix_time) {
    char b[512];
    std::string s = "BEGIN_HEADER\nHDR_VERSION = 1.0\n";
    s += two_row ? "DATATYPE = 4D_SU3_GAUGE\n" : "DATATYPE = 4D_SU3_GAUGE_3x3\n";
    for (int d = 0; d < 4; d++) {
        snprintf(b, sizeof(b), "DIMENSION_%d = %d\n", d + 1, dims[d]);
        s += b;
    }
    snprintf(b, sizeof(b), "CRC32HASH = %x\nCHECKSUM = %x\n", crc32, checksum);
    s += b;
    const char* fmt = two_row ? "%.12g" : "%g";
    std::string num(64, '\0');
    auto g = [&](double x) {
        snprintf(&num[0], num.size(), fmt, x);
        return std::string(num.c_str());
    };
    s += "LINK_TRACE = " + g(link_trace) + "\n";
    s += "PLAQUETTE = " + g(plaquette) + "\n";
    s += "CREATOR = RBC\n";
    const time_t t = (time_t)unix_time;
    char tb[64];
    s += std::string("ARCHIVE_DATE = ") + ctime_r(&t, tb);  // ctime's text ends in a newline
    s += std::string("ENSEMBLE_LABEL = ") + (ensemble_label ? ensemble_label : "") + "\n";
    s += "FLOATING_POINT = IEEE64BIG\nENSEMBLE_ID = NOT yet implemented\n";
    snprintf(b, sizeof(b), "SEQUENCE_NUMBER = %d\n", sequence_number);
    s += b;
    s += "BETA = " + g(beta) + "\n";
    s += "END_HEADER\n";
    return s;
}

uint32_t crc32_register(const uint8_t* p, size_t n) {
    uint32_t tab[256];
    for (uint32_t b = 0; b < 256; b++) {
        uint32_t c = b;
        for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
        tab[b] = c;
    }
    uint32_t c = 0;
    for (size_t i = 0; i < n; i++) c = (c >> 8) ^ tab[(c ^ p[i]) & 0xffu];
    return c;
}

void crc32_shift_tables(size_t nbytes, uint32_t t[4][256]) {
    const ByteTables b(zero_bytes(nbytes));
    memcpy(t, b.t, sizeof(b.t));
}

uint32_t crc32_fold(uint32_t r, const uint32_t* z, size_t n, size_t len_each, size_t len_last) {
    // register(R, A||B) = S_|B|(register(R, A)) ^ register(0, B)
    if (n == 0) return r;
    const ByteTables each(zero_bytes(len_each));
    for (size_t i = 0; i + 1 < n; i++) r = each(r) ^ z[i];
    return (len_last == len_each ? each(r) : ByteTables(zero_bytes(len_last))(r)) ^ z[n - 1];
}

uint32_t crc32_chain(const uint32_t* z, size_t nseg, size_t seg, size_t total) {
    // zlib starts the register at ~0 and complements the result
    if (nseg == 0) return 0u;
    return ~crc32_fold(0xFFFFFFFFu, z, nseg, seg, total - (nseg - 1) * seg);
}

int Pinned::ensure(int nslots, size_t chunk_bytes, std::string& err) {
    if (nslots > kMaxSlots) nslots = kMaxSlots;
    if (slots >= nslots && chunk >= chunk_bytes) return MAG_OK;
    release();
    for (int i = 0; i < nslots; i++) {
        if (cudaHostAlloc(&buf[i], chunk_bytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            release();
            err = "cannot allocate pinned staging buffers";
            return MAG_ERR_NOMEM;
        }
        slots = i + 1;
    }
    chunk = chunk_bytes;
    return MAG_OK;
}

void Pinned::release() {
    for (int i = 0; i < kMaxSlots; i++) {
        if (buf[i]) cudaFreeHost(buf[i]);
        if (ev[i]) cudaEventDestroy(ev[i]);
        buf[i] = nullptr;
        ev[i] = nullptr;
    }
    slots = 0;
    chunk = 0;
}

namespace {

// Ordered chunk pipeline over the pinned ring.  Chunk i uses slot i % K.
// Reading: worker (i mod T) preads chunk i once the copy of chunk i - K out
// of the slot has completed; the caller issues the copies in chunk order.
// Writing: the caller issues the copy of chunk i into its slot once chunk
// i - K has been written; worker (i mod T) pwrites chunk i after its copy.
class Pipeline {
  public:
    Pipeline(Pinned& pin, size_t bytes, int threads, bool to_device)
        : pin_(pin), bytes_(bytes), to_device_(to_device) {
        n_ = (long)((bytes + pin.chunk - 1) / pin.chunk);
        T_ = std::max(1, std::min(threads, pin.slots / 2));
        K_ = std::min(pin.slots, 2 * T_);
        for (int k = 0; k < K_; k++) {
            filled_[k] = -1;
            copied_[k] = -1;
        }
    }

    int run(int fd, long long off, char* dev, cudaStream_t stream, std::string& err) {
        std::vector<std::thread> workers;
        for (int t = 0; t < T_; t++) workers.emplace_back([=] { worker(t, fd, off); });
        int rc = MAG_OK;
        for (long i = 0; i < n_ && rc == MAG_OK; i++) {
            const int k = (int)(i % K_);
            const size_t len = size_of(i);
            if (to_device_) {
                if (!wait_until([&] { return filled_[k] >= i; })) break;  // chunk i in the slot
                if (cudaMemcpyAsync(dev + i * pin_.chunk, pin_.buf[k], len, cudaMemcpyHostToDevice, stream) !=
                        cudaSuccess ||
                    cudaEventRecord(pin_.ev[k], stream) != cudaSuccess)
                    rc = fail_all(MAG_ERR_CUDA, "host to device copy failed");
            } else {
                if (!wait_until([&] { return filled_[k] >= i - K_; })) break;  // chunk i - K written out
                if (cudaMemcpyAsync(pin_.buf[k], dev + i * pin_.chunk, len, cudaMemcpyDeviceToHost, stream) !=
                        cudaSuccess ||
                    cudaEventRecord(pin_.ev[k], stream) != cudaSuccess)
                    rc = fail_all(MAG_ERR_CUDA, "device to host copy failed");
            }
            if (rc == MAG_OK) {
                std::lock_guard<std::mutex> g(m_);
                copied_[k] = i;
                cv_.notify_all();
            }
        }
        for (auto& w : workers) w.join();
        if (rc == MAG_OK && to_device_ && cudaStreamSynchronize(stream) != cudaSuccess)
            rc = fail_all(MAG_ERR_CUDA, "host to device copy failed");
        if (rc == MAG_OK && rc_ != MAG_OK) rc = rc_;
        if (rc != MAG_OK) err = msg_;
        return rc;
    }

  private:
    size_t size_of(long i) const { return i + 1 < n_ ? pin_.chunk : bytes_ - (size_t)i * pin_.chunk; }

    template <typename Pred>
    bool wait_until(Pred p) {
        std::unique_lock<std::mutex> g(m_);
        cv_.wait(g, [&] { return p() || rc_ != MAG_OK; });
        return rc_ == MAG_OK;
    }

    int fail_all(int rc, const char* msg) {
        std::lock_guard<std::mutex> g(m_);
        if (rc_ == MAG_OK) {
            rc_ = rc;
            msg_ = msg;
        }
        cv_.notify_all();
        return rc;
    }

    void worker(int t, int fd, long long off) {
        for (long i = t; i < n_; i += T_) {
            const int k = (int)(i % K_);
            if (to_device_) {
                // the copy of chunk i - K out of this slot was issued; wait for it to finish
                if (i >= K_) {
                    if (!wait_until([&] { return copied_[k] >= i - K_; })) return;
                    if (cudaEventSynchronize(pin_.ev[k]) != cudaSuccess) {
                        fail_all(MAG_ERR_CUDA, "cudaEventSynchronize failed");
                        return;
                    }
                }
                if (!xfer(fd, off + (long long)i * (long long)pin_.chunk, pin_.buf[k], size_of(i), true)) return;
            } else {
                if (!wait_until([&] { return copied_[k] >= i; })) return;
                if (cudaEventSynchronize(pin_.ev[k]) != cudaSuccess) {
                    fail_all(MAG_ERR_CUDA, "cudaEventSynchronize failed");
                    return;
                }
                if (!xfer(fd, off + (long long)i * (long long)pin_.chunk, pin_.buf[k], size_of(i), false)) return;
            }
            std::lock_guard<std::mutex> g(m_);
            filled_[k] = i;
            cv_.notify_all();
        }
    }

    bool xfer(int fd, long long pos, void* b, size_t len, bool read) {
        char* p = static_cast<char*>(b);
        while (len) {
            const ssize_t r = read ? pread(fd, p, len, (off_t)pos) : pwrite(fd, p, len, (off_t)pos);
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) {
                if (read && r == 0) fail_all(MAG_ERR_FORMAT, "payload shorter than the lattice needs");
                else fail_all(MAG_ERR_IO, read ? "read failed" : "write failed");
                return false;
            }
            p += r;
            pos += r;
            len -= (size_t)r;
        }
        return true;
    }

    Pinned& pin_;
    size_t bytes_;
    bool to_device_;
    long n_ = 0;
    int T_ = 1, K_ = 2;
    long filled_[Pinned::kMaxSlots];  // reading: chunk now in the slot; writing: chunk written from it
    long copied_[Pinned::kMaxSlots];  // last chunk whose device copy was issued on the slot
    std::mutex m_;
    std::condition_variable cv_;
    int rc_ = MAG_OK;
    std::string msg_;
};

}  // namespace

int file_to_device(int fd, long long off, void* d, size_t bytes, Pinned& pin, int threads, cudaStream_t stream,
                   std::string& err) {
    if (bytes == 0) return MAG_OK;
    Pipeline p(pin, bytes, threads, true);
    return p.run(fd, off, static_cast<char*>(d), stream, err);
}

int device_to_file(const void* d, size_t bytes, int fd, long long off, Pinned& pin, int threads,
                   cudaStream_t stream, std::string& err) {
    if (bytes == 0) return MAG_OK;
    Pipeline p(pin, bytes, threads, false);
    return p.run(fd, off, const_cast<char*>(static_cast<const char*>(d)), stream, err);
}

}  // namespace nersc
}  // namespace magb

// nersc_host.cpp -- host side of NERSC configuration I/O (see nersc_host.h).
#include "nersc_host.h"

#include <stdlib.h>
#include <string.h>
#include <time.h>

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

uint32_t crc32_chain(const uint32_t* z, size_t nseg, size_t seg, size_t total) {
    // register(R, A||B) = shift_|B|(register(R, A)) ^ register(0, B); zlib starts at ~0 and complements
    uint32_t r = 0xFFFFFFFFu;
    if (nseg == 0) return ~r;
    const ByteTables full(zero_bytes(seg));
    for (size_t i = 0; i + 1 < nseg; i++) r = full(r) ^ z[i];
    const size_t last = total - (nseg - 1) * seg;
    r = (last == seg ? full(r) : ByteTables(zero_bytes(last))(r)) ^ z[nseg - 1];
    return ~r;
}

int Pinned::ensure(size_t chunk_bytes, std::string& err) {
    if (buf[0] && chunk >= chunk_bytes) return MAG_OK;
    release();
    for (int i = 0; i < 2; i++) {
        if (cudaHostAlloc(&buf[i], chunk_bytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            release();
            err = "cannot allocate pinned staging buffers";
            return MAG_ERR_NOMEM;
        }
    }
    chunk = chunk_bytes;
    return MAG_OK;
}

void Pinned::release() {
    for (int i = 0; i < 2; i++) {
        if (buf[i]) cudaFreeHost(buf[i]);
        if (ev[i]) cudaEventDestroy(ev[i]);
        buf[i] = nullptr;
        ev[i] = nullptr;
    }
    chunk = 0;
}

int file_to_device(FILE* f, void* d, size_t bytes, Pinned& pin, cudaStream_t stream, std::string& err) {
    // chunk k is read into buffer k % 2 once the copy of chunk k - 2 out of it has finished
    size_t done = 0;
    for (int k = 0; done < bytes; k++) {
        const int i = k & 1;
        const size_t n = bytes - done < pin.chunk ? bytes - done : pin.chunk;
        if (k >= 2 && cudaEventSynchronize(pin.ev[i]) != cudaSuccess) {
            err = "cudaEventSynchronize failed";
            return MAG_ERR_CUDA;
        }
        if (fread(pin.buf[i], 1, n, f) != n) {
            err = "payload shorter than the lattice needs";
            return MAG_ERR_FORMAT;
        }
        if (cudaMemcpyAsync(static_cast<char*>(d) + done, pin.buf[i], n, cudaMemcpyHostToDevice, stream) !=
                cudaSuccess ||
            cudaEventRecord(pin.ev[i], stream) != cudaSuccess) {
            err = "host to device copy failed";
            return MAG_ERR_CUDA;
        }
        done += n;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) {
        err = "host to device copy failed";
        return MAG_ERR_CUDA;
    }
    return MAG_OK;
}

int device_to_file(const void* d, size_t bytes, FILE* f, Pinned& pin, cudaStream_t stream, std::string& err) {
    // the copy of chunk k overlaps the write of chunk k - 1
    const size_t nchunk = (bytes + pin.chunk - 1) / pin.chunk;
    auto size_of = [&](size_t k) { return k + 1 < nchunk ? pin.chunk : bytes - k * pin.chunk; };
    for (size_t k = 0; k <= nchunk; k++) {
        if (k < nchunk) {
            const int i = (int)(k & 1);
            if (cudaMemcpyAsync(pin.buf[i], static_cast<const char*>(d) + k * pin.chunk, size_of(k),
                                cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaEventRecord(pin.ev[i], stream) != cudaSuccess) {
                err = "device to host copy failed";
                return MAG_ERR_CUDA;
            }
        }
        if (k >= 1) {
            const int j = (int)((k - 1) & 1);
            if (cudaEventSynchronize(pin.ev[j]) != cudaSuccess) {
                err = "device to host copy failed";
                return MAG_ERR_CUDA;
            }
            if (fwrite(pin.buf[j], 1, size_of(k - 1), f) != size_of(k - 1)) {
                err = "write failed";
                return MAG_ERR_IO;
            }
        }
    }
    return MAG_OK;
}

}  // namespace nersc
}  // namespace magb

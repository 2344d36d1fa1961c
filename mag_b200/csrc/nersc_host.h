// nersc_host.h -- host side of NERSC configuration I/O (field-matrix.h:452-713):
// header parsing and formatting, CRC-32 chaining, chunked file <-> device copies.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

namespace magb {
namespace nersc {

// Fields of the header that import_config_nersc reads (field-matrix.h:605-650),
// plus the optional ones export_config_nersc writes.
struct Header {
    std::string datatype;
    int dims[4] = {0, 0, 0, 0};
    bool has_checksum = false;
    uint32_t checksum = 0;
    bool has_plaquette = false;
    double plaquette = 0.0;
    bool has_link_trace = false;
    double link_trace = 0.0;
    bool has_crc32 = false;
    uint32_t crc32 = 0;
    long long payload_offset = -1;  // file offset just after the END_HEADER line
};

// Reads the header with the reference's rules: one line at a time; a line that
// contains a keyword carries its value after the first '=' (blanks and tabs
// skipped, one trailing newline removed); CHECKSUM is hexadecimal; the header
// ends at the first line containing END_HEADER.  Returns MAG_OK, MAG_ERR_IO or
// MAG_ERR_FORMAT (err holds the message).
int read_header(FILE* f, Header& h, std::string& err);

// DATATYPE -> rows stored per link: 4D_SU3_GAUGE -> two_row = 1,
// 4D_SU3_GAUGE_3x3 -> 0; anything else is MAG_ERR_FORMAT.
int datatype_rows(const std::string& datatype, int& two_row, std::string& err);

// The header block export_config_nersc writes (field-matrix.h:486-508 and
// :530-552), keys in the same order; LINK_TRACE, PLAQUETTE and BETA with 12
// significant digits for the two-row type and 6 for 3x3 (the stream precision
// of the reference).
std::string format_header(const int dims[4], int two_row, uint32_t crc32, uint32_t checksum, double link_trace,
                          double plaquette, const char* ensemble_label, int sequence_number, double beta,
                          long long unix_time);

// CRC-32 (zlib) of a byte string from per-segment registers: z[i] is the
// register of segment i started at 0 (no complement), all segments `seg`
// bytes except possibly the last; total = bytes of the string.
uint32_t crc32_chain(const uint32_t* z, size_t nseg, size_t seg, size_t total);
// register of one segment on the host (same definition as the device kernel)
uint32_t crc32_register(const uint8_t* p, size_t n);
// register advance over n zero bytes as four byte tables: S_n(v) = t[0][v & 255] ^ t[1][(v >> 8) & 255] ^ ...
void crc32_shift_tables(size_t nbytes, uint32_t t[4][256]);
// r <- S_len_i(r) ^ z[i] for i = 0..n-1, len_i = len_each except len_last for the last one
uint32_t crc32_fold(uint32_t r, const uint32_t* z, size_t n, size_t len_each, size_t len_last);

// Pinned ring of chunk buffers for pipelined copies between a file and
// device memory: reader/writer threads move chunks between the file (pread /
// pwrite, page cache) and the ring while the calling thread issues the
// host<->device copies in order on the stream.
struct Pinned {
    static constexpr int kMaxSlots = 32;
    void* buf[kMaxSlots] = {};
    cudaEvent_t ev[kMaxSlots] = {};
    int slots = 0;
    size_t chunk = 0;
    int ensure(int nslots, size_t chunk_bytes, std::string& err);
    void release();
};

// file (descriptor fd, payload at byte offset off) -> device memory d, with
// `threads` reader threads; MAG_OK / MAG_ERR_IO / MAG_ERR_FORMAT (short file) / MAG_ERR_CUDA
int file_to_device(int fd, long long off, void* d, size_t bytes, Pinned& pin, int threads, cudaStream_t stream,
                   std::string& err);
// device memory d -> file at byte offset off, with `threads` writer threads
int device_to_file(const void* d, size_t bytes, int fd, long long off, Pinned& pin, int threads,
                   cudaStream_t stream, std::string& err);

}  // namespace nersc
}  // namespace magb

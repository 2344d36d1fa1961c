// mag_nersc_api.cu -- NERSC configuration files (export_config_nersc /
// import_config_nersc): header parsing, the file <-> device pipeline through
// pinned chunks, and the payload's CRC-32, 32-bit checksum and plaquette /
// trace checks on the GPU.  The context is in ctx.h.
#include "ctx.h"

namespace {

constexpr size_t kIoChunk = 8u << 20;      // pinned chunk of the file <-> device copies

// reader / writer threads of the file <-> device pipeline (two pinned slots each)
int io_threads() {
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(2u, std::min(8u, hc / 2));
}

void fill_info(mag_nersc_info* info, const nersc::Header& h, int two_row) {
    memset(info, 0, sizeof(*info));
    for (int d = 0; d < 4; d++) info->dims[d] = h.dims[d];
    info->two_row = two_row;
    info->payload_offset = h.payload_offset;
    info->checksum_header = h.checksum;
    info->crc32_header = h.crc32;
    info->plaquette_header = h.plaquette;
    info->link_trace_header = h.link_trace;
}

struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};

}  // namespace

namespace magb {

int nersc_buffers(mag_ctx* ctx) {
    std::string err;
    int r = ctx->pin.ensure(2 * io_threads(), kIoChunk, err);
    if (r != MAG_OK) return fail(r, err);
    if (!ctx->d_crc) {
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc, sizeof(uint32_t) * (kCrcThreads + 1)));
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc2, sizeof(uint32_t) * (kCrcThreads / kCrcGroup + 1)));
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc_tab, sizeof(uint32_t) * 4 * 256));
        MAG_TRY(ctx->alloc((void**)&ctx->d_csum, sizeof(unsigned int)));
    }
    return MAG_OK;
}

// the CRC-32 shift tables for segments of seg bytes, on the device
int ensure_crc_tab(mag_ctx* ctx, size_t seg) {
    if (ctx->crc_tab_seg == seg) return MAG_OK;
    uint32_t tab[4][256];
    nersc::crc32_shift_tables(seg, tab);
    MAG_CUDA(cudaMemcpyAsync(ctx->d_crc_tab, tab, sizeof(tab), cudaMemcpyHostToDevice, ctx->stream));
    MAG_TRY(ctx->sync("crc tables"));
    ctx->crc_tab_seg = seg;
    return MAG_OK;
}

}  // namespace magb

namespace {

// avg_plaquette (field-matrix.h:387-389) and avg_real_trace (:391-405) of one chain
int plaq_and_trace(mag_ctx* ctx, int chain, double* plaq, double* trace) {
    launch_action_sums<double>(ctx->geom, ctx->U, false, ctx->partial, ctx->sums, SLOT_SCRATCH, SLOT_SCRATCH,
                               ctx->stream);
    launch_link_trace_sum(ctx->geom, ctx->U, ctx->partial, ctx->sums, SLOT_SCRATCH2, ctx->stream);
    MAG_TRY(ctx->check("NERSC plaquette"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const double V = (double)ctx->hc[chain].V;
    const dd2 pl = s[chain * NUM_SLOTS + SLOT_SCRATCH], tr = s[chain * NUM_SLOTS + SLOT_SCRATCH2];
    *plaq = (pl.hi + pl.lo) / (18.0 * V);
    *trace = (tr.hi + tr.lo) / (12.0 * V);
    return MAG_OK;
}

// CRC-32 and 32-bit word sum of the payload in staging, taken in host order:
// on import the big-endian payload is converted to host order first, on export
// it is converted to big-endian afterwards
int payload_digest(mag_ctx* ctx, size_t bytes, bool import, uint32_t* crc, uint32_t* csum) {
    const size_t seg = crc_seg(bytes);
    const size_t nfull = bytes / seg, tail = bytes - nfull * seg;
    const size_t ngroups = (nfull + kCrcGroup - 1) / kCrcGroup;
    MAG_TRY(ensure_crc_tab(ctx, seg));
    MAG_CUDA(cudaMemsetAsync(ctx->d_csum, 0, sizeof(unsigned int), ctx->stream));
    if (import) launch_swap64_sum32(ctx->staging, bytes, true, ctx->d_csum, ctx->stream);
    launch_crc32_segments(ctx->staging, bytes, seg, ctx->d_crc, ctx->stream);
    launch_crc32_fold(ctx->d_crc, nfull, kCrcGroup, ctx->d_crc_tab, ctx->d_crc2, ctx->stream);
    if (!import) launch_swap64_sum32(ctx->staging, bytes, false, ctx->d_csum, ctx->stream);
    MAG_TRY(ctx->check("NERSC payload digest"));
    std::vector<uint32_t> z2(ngroups + 1);
    unsigned int sum = 0;
    if (ngroups)
        MAG_CUDA(cudaMemcpyAsync(z2.data(), ctx->d_crc2, sizeof(uint32_t) * ngroups, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    if (tail)
        MAG_CUDA(cudaMemcpyAsync(&z2[ngroups], ctx->d_crc + nfull, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MAG_CUDA(cudaMemcpyAsync(&sum, ctx->d_csum, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    MAG_TRY(ctx->sync("NERSC payload digest"));
    // zlib: register started at ~0, result complemented; groups of kCrcGroup segments, the last group shorter
    uint32_t r = 0xFFFFFFFFu;
    if (ngroups) {
        const size_t last = (nfull - (ngroups - 1) * kCrcGroup) * seg;
        r = nersc::crc32_fold(r, z2.data(), ngroups, kCrcGroup * seg, last);
    }
    if (tail) r = nersc::crc32_fold(r, &z2[ngroups], 1, tail, tail);
    *crc = ~r;
    *csum = sum;
    return MAG_OK;
}

}  // namespace

extern "C" {

int mag_nersc_read_header(const char* path, mag_nersc_info* info) {
    if (!path || !info) return fail(MAG_ERR_ARG, "mag_nersc_read_header: null argument");
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(MAG_ERR_IO, std::string("cannot open ") + path);
    nersc::Header h;
    std::string err;
    int two_row = 0;
    int r = nersc::read_header(fc.f, h, err);
    if (r == MAG_OK) r = nersc::datatype_rows(h.datatype, two_row, err);
    if (r != MAG_OK) return fail(r, std::string("import_config_nersc: ") + err);
    fill_info(info, h, two_row);
    return MAG_OK;
}

int mag_gauge_load_nersc(mag_ctx* ctx, int chain, const char* path, mag_nersc_info* info) {
    if (!ctx || !path) return fail(MAG_ERR_ARG, "mag_gauge_load_nersc: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(MAG_ERR_IO, std::string("cannot open ") + path);
    nersc::Header h;
    std::string err;
    int two_row = 0;
    int r = nersc::read_header(fc.f, h, err);
    if (r == MAG_OK) r = nersc::datatype_rows(h.datatype, two_row, err);
    if (r != MAG_OK) return fail(r, std::string("import_config_nersc: ") + err);
    for (int d = 0; d < 4; d++)
        if (h.dims[d] != ci.L[d])
            return fail(MAG_ERR_FORMAT, "import_config_nersc: WRONG Lattice Size (file " + std::to_string(h.dims[0]) +
                                            "x" + std::to_string(h.dims[1]) + "x" + std::to_string(h.dims[2]) + "x" +
                                            std::to_string(h.dims[3]) + ")");
    MAG_TRY(nersc_buffers(ctx));
    const size_t bytes = (size_t)ci.V * 4 * (two_row ? 6 : 9) * 16;
    r = nersc::file_to_device(fileno(fc.f), h.payload_offset, ctx->staging, bytes, ctx->pin, io_threads(),
                              ctx->stream, err);
    if (r != MAG_OK) return fail(r, "import_config_nersc: " + err);
    uint32_t crc = 0, csum = 0;
    MAG_TRY(payload_digest(ctx, bytes, true, &crc, &csum));
    if (info) {
        fill_info(info, h, two_row);
        info->checksum = csum;
        info->crc32 = crc;
    }
    // field-matrix.h:673-676 / :695-699: the links are left untouched on a checksum mismatch
    if (csum != h.checksum) {
        char b[128];
        snprintf(b, sizeof(b), "import_config_nersc: WRONG Checksum: %x(labeled) vs %x(computed)", h.checksum, csum);
        return fail(MAG_ERR_CHECKSUM, b);
    }
    launch_payload_to_links(ctx->staging, two_row, ci.off, ci.V, ctx->U, ctx->stream);
    MAG_TRY(ctx->refresh_copy());
    double plaq = 0.0, trace = 0.0;
    MAG_TRY(plaq_and_trace(ctx, chain, &plaq, &trace));
    if (info) {
        info->plaquette = plaq;
        info->link_trace = trace;
    }
    // field-matrix.h:708-711
    if (std::fabs(plaq - h.plaquette) > 1e-4) {
        char b[160];
        snprintf(b, sizeof(b), "import_config_nersc: Plaquette: %.8f(labeled) vs %.8f(computed)", h.plaquette, plaq);
        return fail(MAG_ERR_PLAQUETTE, b);
    }
    return MAG_OK;
}

int mag_gauge_save_nersc(mag_ctx* ctx, int chain, const char* path, int two_row, double beta,
                         int sequence_number, const char* ensemble_label, mag_nersc_info* info) {
    if (!ctx || !path) return fail(MAG_ERR_ARG, "mag_gauge_save_nersc: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    MAG_TRY(nersc_buffers(ctx));
    double plaq = 0.0, trace = 0.0;
    MAG_TRY(plaq_and_trace(ctx, chain, &plaq, &trace));
    const size_t bytes = (size_t)ci.V * 4 * (two_row ? 6 : 9) * 16;
    launch_links_to_payload(ctx->U, two_row ? 1 : 0, ci.off, ci.V, ctx->staging, ctx->stream);
    uint32_t crc = 0, csum = 0;
    MAG_TRY(payload_digest(ctx, bytes, false, &crc, &csum));
    const std::string hdr = nersc::format_header(ci.L, two_row ? 1 : 0, crc, csum, trace, plaq, ensemble_label,
                                                 sequence_number, beta, (long long)time(nullptr));
    const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return fail(MAG_ERR_IO, std::string("cannot create ") + path);
    std::string err;
    int r = MAG_OK;
    if (pwrite(fd, hdr.data(), hdr.size(), 0) != (ssize_t)hdr.size()) {
        r = MAG_ERR_IO;
        err = "header write failed";
    }
    if (r == MAG_OK)
        r = nersc::device_to_file(ctx->staging, bytes, fd, (long long)hdr.size(), ctx->pin, io_threads(),
                                  ctx->stream, err);
    if (close(fd) != 0 && r == MAG_OK) {
        r = MAG_ERR_IO;
        err = "close failed";
    }
    if (r != MAG_OK) return fail(r, "export_config_nersc: " + err);
    if (info) {
        memset(info, 0, sizeof(*info));
        for (int d = 0; d < 4; d++) info->dims[d] = ci.L[d];
        info->two_row = two_row ? 1 : 0;
        info->payload_offset = (int64_t)hdr.size();
        info->checksum_header = info->checksum = csum;
        info->crc32_header = info->crc32 = crc;
        info->plaquette_header = info->plaquette = plaq;
        info->link_trace_header = info->link_trace = trace;
    }
    return MAG_OK;
}

int mag_crc32_host(const void* data, size_t n, size_t seg, uint32_t* crc) {
    if ((!data && n) || !crc || seg == 0 || seg % 16) return fail(MAG_ERR_ARG, "mag_crc32_host: bad argument");
    const uint8_t* p = static_cast<const uint8_t*>(data);
    const size_t nseg = (n + seg - 1) / seg;
    std::vector<uint32_t> z(nseg);
    for (size_t i = 0; i < nseg; i++) z[i] = nersc::crc32_register(p + i * seg, std::min(seg, n - i * seg));
    *crc = nersc::crc32_chain(z.data(), nseg, seg, n);
    return MAG_OK;
}

}  // extern "C"


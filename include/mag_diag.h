/*
 * mag_diag.h -- measurement entry points of libmag_b200.so.
 *
 * These have no counterpart in the reference (which only has qlat's TIMER()
 * scoped timers, field-hmc.h:341 / :903); they exist for benchmarking and
 * roofline accounting.  All times are CUDA-event times on the context's stream.
 */
#ifndef MAG_DIAG_H
#define MAG_DIAG_H

#include "mag_c.h"

#ifdef __cplusplus
extern "C" {
#endif

/* device time of the trajectories of the last mag_run call (ms) */
int mag_last_run_ms(mag_ctx* ctx, double* total_ms);
/* device time of the kernels of the last mag_wilson_loops call (ms) */
int mag_last_measure_ms(mag_ctx* ctx, double* ms);
/* average device time of one force evaluation (thin or smeared, in the
   context's precision, constraint fix-up included) on the current links */
int mag_time_force(mag_ctx* ctx, int reps, double* ms_per_eval);
/* average device time of one launch of a single kernel on the current
   fields: "force", "staple", "stout_forward", "stout_lambda", "stout_chain",
   "evolve", "kick", "action", and the NERSC payload kernels on chain 0's
   3x3 payload made from the current links: "nersc_swap" (byte order +
   word checksum), "nersc_crc" (segment CRC-32), "nersc_to_links",
   "nersc_from_links", "nersc_plaq" (plaquette and link-trace sums) */
int mag_time_kernel(mag_ctx* ctx, const char* which, int reps, double* ms_per_launch);
/* re-run the launch-configuration tuner: time every variant of the staple /
   force / stout kernels on the live fields (`reps` launches each) and keep the
   fastest.  Variants: one thread per link at minimum blocks per SM 2..5
   ("t1m2".."t1m5", register caps), and for the staple, force and chain-rule
   kernels the direction split "s<NS>r<R>" (NS = 3 or 6 warps per 32-link tile,
   register cap R).  Every variant is timed; the choice is made among the
   one-thread-per-link variants, which give bit-identical results (the split
   shapes sum in another order and are selected only by mag_set_kernel_variant).
   The tuner then times whole force evaluations with the link kernels' blocks
   visiting a single lattice in raster order or in 2 x 2 / 4 x 4 tiles of
   (x2, x3) rows (same results, other L2 reuse) and keeps the fastest order.
   report (may be NULL) receives a JSON object
   {"family": {"fp64": [chosen, {variant: ms, ...}], "fp32": [...]}, ...,
    "block_order": [tile, {"raster": ms, "tile2": ms, "tile4": ms}]}
   (times only for the families and precisions the context tuned).  The first
   trajectory, integration or graph build of a context runs the tuner once. */
int mag_autotune(mag_ctx* ctx, int reps, char* report, size_t len);
/* use `variant` (a name as in the mag_autotune report) for kernel `family`
   ("force", "staple", "stout_forward", "stout_lambda", "stout_chain") at
   precision 0 (FP64) or 1 (FP32) from now on, in place of the tuner's choice */
int mag_set_kernel_variant(mag_ctx* ctx, const char* family, int precision, const char* variant);
/* number of kernel nodes in the captured trajectory graph (building it if needed) */
int mag_graph_kernel_count(mag_ctx* ctx, int* kernels);
/* measured CUDA-core FMA throughput of this device: precision 0 = FP64 FMA,
   1 = FP32 FMA, 2 = packed FP32 FMA (fma.rn.f32x2), 3 = packed FP32 FMA whose
   operands are formed every iteration by swapping, negating one half of and
   broadcasting changing pairs; tflops counts 2 flops per FMA */
int mag_probe_fma_peak(int precision, double* tflops);
/* CRC-32 (zlib) of n host bytes computed the way NERSC export/import does on
   the device: seg-byte segment registers (seg a multiple of 16) chained with
   the zero-byte shift; host only (tests the chaining without a GPU) */
int mag_crc32_host(const void* data, size_t n, size_t seg, uint32_t* crc);

#ifdef __cplusplus
}
#endif
#endif /* MAG_DIAG_H */

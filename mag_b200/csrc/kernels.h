// kernels.h -- host-side launchers of the sm_100a kernels (no torch types).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.cuh"

namespace magb {

struct dd2 {
    double hi, lo;
};

// Geometry shared by every launch of a context.
struct DevGeom {
    const ChainInfo* chains;   // device array [nchain]
    const uint16_t* c2c;       // device array [vpad / MAG_CHUNK]
    long vpad;                 // padded global sites (multiple of MAG_CHUNK)
    int nchain;
    // device array [nchain]: the chain's Philox stream index, added to a seed to form its
    // key (default: the chain's position in the context; a sharded ensemble sets the
    // chain's position in the whole ensemble)
    const unsigned long long* stream_index;
    // Order in which the link kernels' 128-site blocks visit a single lattice:
    // tile = 0 raster (x0 fastest); tile = T > 0: the (x2, x3) rows in T x T
    // tiles, rows of `gpr` blocks (x0 x1 = 128 gpr sites), L2 rows along x2.
    // Only the order changes: every link is computed as in raster order.
    int tile, gpr, L2;
};

// Per-trajectory record kept on the device, one per chain per trajectory.
struct TrajRecord {
    double h_old, h_new, delta_h;
    double kin_old, kin_new, pot_old, pot_new;
    double plaq_old, plaq_new, rect_old, rect_new;
    double uniform;
    double demon0, demon1;
    double reunit_maxdev;
    double avg_plaquette;
    int accept;
    int traj;
};

// Device-resident state of the accept step of one chain.
struct ChainState {
    double demon0, demon1;
    int accept;
    int naccept;
};

// Slots of the per-chain double-double sums
enum SumSlot {
    SLOT_PLAQ_OLD = 0, SLOT_RECT_OLD, SLOT_KIN_OLD,
    SLOT_PLAQ_NEW, SLOT_RECT_NEW, SLOT_KIN_NEW,
    SLOT_PLAQ_THIN, SLOT_RECT_THIN, SLOT_SCRATCH, SLOT_SCRATCH2,
    NUM_SLOTS
};

struct AcceptArgs {
    int metropolis;          // 1 Metropolis, 0 demon
    int action_iwasaki;
    double e_max;
    int n_forced;
    const double* uniform_override;  // nullptr: Philox(seed + chain, traj)
    unsigned long long seed;
};

// ---- force and staples (kernels_force.cu)
// `v` selects the register-cap variant 0..3 (minimum 2..5 resident 128-thread
// blocks per SM, i.e. at most 255 / 168 / 128 / 102 registers per thread).
constexpr int kForceBlockSites = 128;  // sites per block of the one-thread-per-link kernels
constexpr int kNumRegVariants = 4;  // one thread per link, register caps (minimum blocks per SM 2..5)
constexpr int kNumVariants = 9;     // + direction split: 3 or 6 warps per 32-link tile, register caps
enum KernelFamily { KF_FORCE = 0, KF_STAPLE, KF_STOUT_FWD, KF_STOUT_LAMBDA, KF_STOUT_CHAIN, KF_COUNT };

// W = double links U(x,mu) U(x+mu,mu); the Iwasaki staple kernels read W of the same field
template <typename T>
void launch_double_link(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, cudaStream_t s);
template <typename T>
void launch_force(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, AlgPlanes<T> F, bool iwasaki, int v,
                  cudaStream_t s);
template <typename T>
void launch_staple_dagger(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, LinkPlanes<T> Z, bool iwasaki, int v,
                          cudaStream_t s);
template <typename T>
void launch_constraint_fixup(const DevGeom& g, LinkPlanes<T> U, AlgPlanes<T> F, cudaStream_t s);
template <typename T>
void launch_stout_forward(const DevGeom& g, LinkPlanes<T> Uin, LinkPlanes<T> Uout, AlgPlanes<T> Q, int v,
                          cudaStream_t s);
template <typename T>
void launch_stout_lambda(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Q, LinkPlanes<T> Z, AlgPlanes<T> Lam,
                         LinkPlanes<T> Zp, int v, cudaStream_t s);
template <typename T>
void launch_stout_chain(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp, LinkPlanes<T> Zout,
                        int v, cudaStream_t s);
template <typename T>
void launch_stout_chain_force(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp, AlgPlanes<T> F,
                              int v, cudaStream_t s);

// ---- streaming kernels (kernels_update.cu)
template <typename TU, typename TX>
void launch_evolve(const DevGeom& g, LinkPlanes<TU> Uin, LinkPlanes<TU> Uout, AlgPlanes<TX> X, double eps,
                   LinkPlanes<float> Ucopy, cudaStream_t s);
template <typename TF>
void launch_kick(const DevGeom& g, AlgPlanes<double> P, AlgPlanes<TF> F, double eps, cudaStream_t s);
// reunit[chain] receives the max deviation as double bits (caller zeroes it first)
void launch_reunitarize(const DevGeom& g, LinkPlanes<double> U, LinkPlanes<float> Ucopy,
                        unsigned long long* reunit, cudaStream_t s);
void launch_copy_to_float(const DevGeom& g, LinkPlanes<double> U, LinkPlanes<float> U32, cudaStream_t s);
void launch_link_copy(const DevGeom& g, LinkPlanes<double> src, LinkPlanes<double> dst, cudaStream_t s);
void launch_restore_rejected(const DevGeom& g, LinkPlanes<double> backup, LinkPlanes<double> U,
                             LinkPlanes<float> U32, const ChainState* st, cudaStream_t s);

// ---- reductions (kernels_update.cu); partial must hold vpad / MAG_CHUNK * 2 dd2
template <typename T>
void launch_action_sums(const DevGeom& g, LinkPlanes<T> U, bool with_rect, dd2* partial, dd2* sums, int slot_plaq,
                        int slot_rect, cudaStream_t s);
void launch_kinetic_sum(const DevGeom& g, AlgPlanes<double> P, dd2* partial, dd2* sums, int slot, cudaStream_t s);
void launch_accept(const DevGeom& g, const AcceptArgs& a, dd2* sums, ChainState* st,
                   const unsigned long long* reunit, TrajRecord* rec, long long* traj_counter, cudaStream_t s);
// completes rec[] with the thin plaquette, appends it to hist[(counter - *hist_base) * nchain + c]
// when that index is below hist_cap, then advances the trajectory counter
void launch_record_plaquette(const DevGeom& g, const dd2* sums, TrajRecord* rec, TrajRecord* hist,
                             const long long* hist_base, int hist_cap, long long* traj_counter, cudaStream_t s);

// ---- RNG and layout (kernels_update.cu)
void launch_momenta(const DevGeom& g, AlgPlanes<double> P, unsigned long long seed, const long long* traj_counter,
                    cudaStream_t s);
void launch_hot_start(const DevGeom& g, LinkPlanes<double> U, unsigned long long seed, cudaStream_t s);
void launch_cold_start(const DevGeom& g, LinkPlanes<double> U, cudaStream_t s);
void launch_aos_to_links(const double* aos, int chain_off, int V, LinkPlanes<double> U, long vpad_unused,
                         cudaStream_t s);
void launch_links_to_aos(LinkPlanes<double> U, int chain_off, int V, double* aos, cudaStream_t s);
template <typename T>
void launch_aos_to_alg(const double* aos, int chain_off, int V, AlgPlanes<T> X, cudaStream_t s);
template <typename T>
void launch_alg_to_aos(AlgPlanes<T> X, int chain_off, int V, double* aos, cudaStream_t s);
template <typename T>
void launch_links_to_aos_t(LinkPlanes<T> U, int chain_off, int V, double* aos, cudaStream_t s);

// ---- FMA throughput probe: nblocks x 256 threads, 8 x iters FMAs each
template <typename T>
void launch_fma_probe(T* out, int nblocks, int iters, cudaStream_t s);
// packed FP32 (fma.rn.f32x2): out holds nblocks * 256 float2
void launch_ffma2_probe(void* out, int nblocks, int iters, bool selected_operands, cudaStream_t s);

// sums[c][slot] = sum over the chain's links of ReTr U (avg_real_trace, field-matrix.h:391-405, times 12 V)
void launch_link_trace_sum(const DevGeom& g, LinkPlanes<double> U, dd2* partial, dd2* sums, int slot,
                           cudaStream_t s);

// ---- NERSC payload (kernels_nersc.cu); payload = one chain's links in file order,
// bytes a multiple of 16, 16-byte aligned
// in place: big-endian <-> host order; *sum += 32-bit word sum of the host-order payload
void launch_swap64_sum32(void* payload, size_t bytes, bool to_host, unsigned int* sum, cudaStream_t s);
// z[i] = CRC-32 register (zlib polynomial, zero start, no final complement) of bytes [i*seg, (i+1)*seg)
// of the payload; seg a multiple of 16
void launch_crc32_segments(const void* payload, size_t bytes, size_t seg, uint32_t* z, cudaStream_t s);
// z2[g] = fold of z[g*G .. (g+1)*G) (n registers of equal-length segments) with the one-segment zero-byte
// advance given as four 256-entry byte tables in device memory (tab[k * 256 + b])
void launch_crc32_fold(const uint32_t* z, size_t n, int G, const uint32_t* tab, uint32_t* z2, cudaStream_t s);
// host-order payload <-> links of the chain at site offset off (two_row: 6 complex per link, third row
// rebuilt by reunitarize; else 9)
void launch_payload_to_links(const double* payload, int two_row, int off, int V, LinkPlanes<double> U,
                             cudaStream_t s);
void launch_links_to_payload(LinkPlanes<double> U, int two_row, int off, int V, double* payload, cudaStream_t s);

// ---- single-matrix operators, batched (kernels_matrix.cu): n matrices of 9 complex doubles each,
// row-major, on the device; Q Hermitian traceless (its independent entries are read)
void launch_expiq(const double* q, long n, double* out, cudaStream_t s);
void launch_dexpiq(const double* q, const double* dq, long n, double* out, cudaStream_t s);
void launch_compute_lambda(const double* q, const double* sigma, const double* u, long n, double* lam,
                           cudaStream_t s);

// ---- per-link demon sweep (kernels_demon.cu)
constexpr int kDemonPaths = 168;   // staple paths per link: 6 plaquette, 18 rectangle, 72 chair, 72 twist
constexpr int kDemonWindow = 384;  // capacity of the per-site link window (353 used)
struct DemonState {
    double E[4];  // plaquette, rectangle, chair, twist demons
    long long accept, reject;
};
// The staple paths of the four links of a site as steps through a window of links around the
// site: packed[n] = site offset of slot n (4 bits per coordinate, biased by 4) | direction << 16
// (direction 4: the unit matrix that pads the three-link plaquette paths); step i of path p of
// the link in direction mu reads slot[mu][p][i], as the link (fwd = 1) or its adjoint (fwd = 0)
struct DemonTables {
    int nslot;
    int packed[kDemonWindow];
    uint16_t slot[4][kDemonPaths][5];
    uint8_t fwd[4][kDemonPaths][5];
};
// false if the path set does not fit the window (cannot happen for the fixed path set)
bool build_demon_tables(DemonTables* out);
// One sweep of one chain: its links in the host AoS layout double[V][4][3][3][2] start at
// double2 aos_off of the AoS buffer; its Philox draws use the key `seed`.
struct DemonJob {
    ChainInfo ci;
    long long aos_off;
    unsigned long long seed;
};
// one sweep of each of njobs chains, one CTA per chain (links in site order inside a chain,
// the chains side by side); states[j] holds chain j's demons and hit counts
void launch_demon_sweeps(const DemonJob* jobs, int njobs, double* aos, const DemonTables* tabs, int sweep,
                         double e_max, DemonState* states, cudaStream_t s);

// ---- measurements (kernels_wloop.cu)
// planar R x T loops: lines = Rmax single-direction planes, tl/tl2 = two more;
// out[((i * Tmax + T-1) * nchain + c) * Rmax + R-1] (i = spatial direction)
void launch_wilson_planar(const DevGeom& g, LinkPlanes<double> U, int Rmax, int Tmax, LinkPlanes<double> lines,
                          LinkPlanes<double> tl, LinkPlanes<double> tl2, dd2* partial, dd2* out, cudaStream_t s);
// sum over sites (coarse sites x = 0 mod coarse_mag when coarse_mag > 0) and
// npath closed paths of ReTr; dirs[npath][plen], 0..3 forward, 4..7 backward,
// -1 ends a shorter path; out[c]
void launch_wilson_general(const DevGeom& g, LinkPlanes<double> U, const int* dirs, int npath, int plen,
                           int coarse_mag, dd2* partial, dd2* out, cudaStream_t s);

// ---- two-level coupling (kernels_multi.cu), FP64; cf / cc the fine and coarse chain (one each, off 0).
// Coarse links: energy density ReTr(C^dag e^{iQ} V) reduced into *energy (partial: 4 * ceil(Vc / 128)
// dd2; both may be null), the coarse force into Fc, Lambda and C^dag e^{iQ} into Lam / Zp (each may be null).
void launch_multi_coarse(const ChainInfo& cf, const ChainInfo& cc, LinkPlanes<double> U, LinkPlanes<double> C,
                         double rho, double eta_sqr, AlgPlanes<double> Fc, AlgPlanes<double> Lam, LinkPlanes<double> Zp,
                         dd2* partial, dd2* energy, cudaStream_t s);
// F += the coupling's derivative with respect to the fine links (needs Lam, Zp of the same fields)
void launch_multi_fine(const ChainInfo& cf, const ChainInfo& cc, LinkPlanes<double> U, AlgPlanes<double> Lam,
                       LinkPlanes<double> Zp, double rho, double eta_sqr, AlgPlanes<double> F, cudaStream_t s);

}  // namespace magb

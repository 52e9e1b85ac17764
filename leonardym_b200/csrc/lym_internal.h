// Host-side internal interfaces of the library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lym_common.cuh"

namespace lym {

enum Prec : int { PREC_D = 0, PREC_F = 1, PREC_H = 2 };
enum Rep : int { REP_SU3 = 0, REP_SU2ADJ = 1 };

// A device spinor: full lattice (nparity = 2) or one parity (nparity = 1).
struct Spinor {
    int prec = PREC_D;
    int nparity = 0;
    int stride = 0;
    void *v = nullptr;
    float *norm = nullptr;  // FP16 only
    bool owned = false;

    SpinorD d(int p = 0) const { return SpinorD{(double2 *)v, stride}.par(p); }
    SpinorF f(int p = 0) const { return SpinorF{(float4 *)v, stride}.par(p); }
    SpinorH h(int p = 0) const { return SpinorH{(int4 *)v, norm, stride}.par(p); }
    size_t bytes_per_parity() const;
    // view of one parity of a full spinor
    Spinor parity(int p) const;
};

struct GaugeDev {
    int rep = REP_SU3;
    void *d64 = nullptr;       // FP64: double2[2][4][9][stride] (SU3) or double[2][4][9][stride] (adjoint)
    void *f32 = nullptr;       // FP32 reconstructed: float4[2][4][3][stride] or float2[2][4][3][stride]
    void *h16 = nullptr;       // FP16 reconstructed: uint2[2][4][3][stride] or half2[2][4][3][stride]
    uint8_t *sign = nullptr;   // [2][stride]
    // FP32 SU(3) links in 8 reals (GaugeF8): float4[2][4][2][stride]; link_reals 12 or 8 picks
    // the format of the FP32 single-RHS stencils (lym_set_link_format)
    void *f32r8 = nullptr;
    // FP32 SU(3) links in all 18 reals for the batched stencil (GaugeF18P):
    // float4[2][4][5][stride], the boundary sign included
    void *f32r18 = nullptr;
    int link_reals = 12;
    bool recon_ok = false;
};

struct CloverDev {
    void *T[3] = {nullptr, nullptr, nullptr};     // per precision, [2 parity][2 block][words][stride]
    void *Tinv[3] = {nullptr, nullptr, nullptr};
};

enum Epi : int { EPI_SCALE_ = 0, EPI_CLOVINV_ = 1, EPI_XPAY_ = 2, EPI_XPAY_INV_ = 3, EPI_XPAY_RES_ = 4, EPI_XPAY_OMEGA_ = 5 };

struct DslashParams {
    Geom g;
    int prec = PREC_D;
    int rep = REP_SU3;
    int epi = EPI_SCALE_;
    int parity = 0;          // output parity
    Spinor in;               // view of the input parity (1 - parity)
    Spinor out;              // view of the output parity
    Spinor y;                // same-parity input (EPI_XPAY, EPI_XPAY_INV)
    Spinor v2;               // optional added vector (EPI_XPAY)
    int has_v2 = 0;
    const GaugeDev *U = nullptr;
    const void *clover = nullptr;  // T (EPI_XPAY) or Tinv (EPI_CLOVINV, EPI_XPAY_INV) of this precision
    int gamma5 = 0;
    double a = 1.0, b = 0.0, alpha_re = 0.0, alpha_im = 0.0;
    const int *skip_if = nullptr;
};

// kernels (lym_kernels.cu)
void launch_dslash(const DslashParams &P, cudaStream_t st);
// the second Schur launch of the even-odd CG on (gamma5 S)^2 with its vector work fused
// (mode CG_NORM / CG_UPDATE of lym_dslash.cuh); p, x, r: one parity; state: the CGState;
// partials: one double per block of the launch
void launch_dslash_cg(const DslashParams &P, int mode, const Spinor &p, const Spinor &x, const Spinor &r, void *state,
                      double *partials, unsigned int *counter, cudaStream_t st);
void launch_clover(const Geom &g, int prec, const Spinor &out, const Spinor &in, const void *clover, int parity,
                   int gamma5, cudaStream_t st);
void launch_pack(const Geom &g, const double *aos, const Spinor &full, cudaStream_t st);
void launch_unpack(const Geom &g, const Spinor &full, double *aos, cudaStream_t st);
void launch_upload_gauge(const Geom &g, int rep, const double *aos, GaugeDev &U, cudaStream_t st);
void launch_compress_gauge(const Geom &g, GaugeDev &U, int *err, cudaStream_t st);
void launch_fundamental_to_fermion(const Geom &g, int rep, int bc, const double *gauge_aos, double *fermion_aos,
                                   cudaStream_t st);
void launch_clover_build(const Geom &g, const GaugeDev &U, double kc, CloverDev &C, double *F_aos, int *err,
                         cudaStream_t st);
void launch_clover_compress(const Geom &g, CloverDev &C, cudaStream_t st);
void launch_neighbour_tables(const Geom &g, int *sup, int *sdn, cudaStream_t st);
void launch_stencil_index_probe(const Geom &g, int *out, cudaStream_t st);
void launch_convert(const Geom &g, const Spinor &dst, const Spinor &src, cudaStream_t st);

}  // namespace lym

namespace lym {
// A batch of nb right-hand sides of one parity, interleaved (see lym_batch.cuh).
struct SpinorBatch {
    int prec = PREC_F;   // PREC_F or PREC_H
    int nb = 0, lognb = 0, stride = 0;
    void *v = nullptr;
    float *norm = nullptr;
};

struct DslashBatchParams {
    Geom g;
    int prec = PREC_F, rep = REP_SU3, epi = EPI_SCALE_, parity = 0, gamma5 = 0;
    SpinorBatch in, out, y;
    const GaugeDev *U = nullptr;
    int has_clover = 0;
    double a = 1.0, b = 0.0;
    const int *skip_if = nullptr;
    const int *active = nullptr;
    const int *nbr = nullptr;                  // neighbour table [2][8][stride]
    const int *order = nullptr;                // traversal table [stride] or nullptr (h order)
    int walk_by = 0, walk_bz = 0;              // the column of that traversal (0: h order)
    int minb = 1;                              // kernel variant: minimum resident blocks per SM
    const double *b_slot = nullptr;            // device array [nb] or nullptr
    const void *const *clover_slot = nullptr;  // device array [nb] of FP32 clover bases (T or Tinv)
    const int *uniform = nullptr;              // device flag: every slot on one operator
    // EPI_XPAY_RES: s = r - alpha out with r FP32, s in the precision of out, alpha per RHS
    SpinorBatch res_r, res_s;
    const double2 *res_alpha = nullptr;
    // EPI_XPAY_OMEGA (staged kernel variants only): rhat (FP32) and the per-block partial sums
    // [block][nb][7] of <out, y>, |out|^2, <rhat, y>, <rhat, out>
    SpinorBatch om_rhat;
    double *om_partials = nullptr;
    int *err = nullptr;  // bulk-copy variants: set to 1 when a copy wait gave up
};
// blocks of the batched stencil launch (the size of the EPI_XPAY_OMEGA partials)
inline long batch_stencil_blocks(const Geom &g, int lognb) { return (((long)g.Vh << (lognb - 1)) + 127) / 128; }

void launch_dslash_batch(const DslashBatchParams &P, cudaStream_t st);
// lym_multiply_device_noalloc (lym_noalloc.cu): half-sites of its fixed scratch array, the
// lattice size limit of that entry point (V <= 2 * kNoallocMaxHalfSites, e.g. 16^3 x 32)
constexpr int kNoallocMaxHalfSites = 65536;
// the even-odd operator on AoS device vectors through that array; returns a LYM_* status
// and, on LYM_ERR_CUDA, the CUDA error it saw in *cuda_err
int noalloc_schur(const Geom &g, int rep, int device, cudaStream_t st, const GaugeDev &U, const CloverDev *C,
                  double kappa, int gamma5, double *out, const double *in, cudaError_t *cuda_err);
// the BiCGStab omega sums fused into the second stencil launch of a block Schur product
// (EPI_XPAY_OMEGA_): the variants that support it, the scratch it needs (per-block partial
// sums, then chunk sums) and the launches that add them up and apply the omega update
bool batch_omega_fusable(int minb, int prec);
long omega_scratch_doubles(const Geom &g, int lognb);
void launch_omega_finalize(double *scratch, const Geom &g, int lognb, void *state, cudaStream_t st);
void launch_nbr_table(const Geom &g, int *nbr, cudaStream_t st);
// traversal of the half-sites in by * bz columns of the (y, z) plane, t fastest
// (by | Ly, bz | Lz)
void launch_order_table(const Geom &g, int by, int bz, int *order, cudaStream_t st);
extern const int kBatchMinBlocks[];  // the compiled variants of the batched stencil
extern const int kBatchMinBlocksCount;
extern const int kBatchTunedCount;  // the leading entries the autotuner times

// measurements on AoS spinors in device memory (lym_measure.cu)
struct MesonProps {
    const double2 *p[12];  // the propagator of the point source of spin a, colour c at c * 4 + a
};
constexpr int kMaxDots = 64;
struct DotPairs {
    const double2 *a[kMaxDots];
    const double2 *b[kMaxDots];
};
size_t meson_scratch_bytes(const Geom &g);
// result: [3][Lt] per time slice sums (pion, scalar, PS)
void launch_meson_contractions(const Geom &g, const MesonProps &P, double *scratch, double *result, cudaStream_t st);
int dot_blocks(const Geom &g);
void launch_dots(const Geom &g, const DotPairs &D, int n, int gamma5, double2 *partials, double2 *out,
                 cudaStream_t st);
// force[x][mu] -= sum_i w_i F_mu(x; X_i, Y_i) of the Wilson (clover = 0) or Wilson-clover fermion
// force; X, Y, weights: device arrays of n entries
// scratch: fermion_force_scratch_bytes (the per-site plane matrices of the clover part)
size_t fermion_force_scratch_bytes(const Geom &g);
void launch_fermion_force(const Geom &g, const GaugeDev &U, int n, const double2 *const *X, const double2 *const *Y,
                          const double *weights, double kappa, double csw, int clover, double2 *force,
                          double2 *scratch, cudaStream_t st);
// real Z2 noise vector `stream` of generator `seed` (AoS full spinor)
void launch_z2_noise(const Geom &g, double *out, unsigned long long seed, unsigned long long stream, cudaStream_t st);
}  // namespace lym

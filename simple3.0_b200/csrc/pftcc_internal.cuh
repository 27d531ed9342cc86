// pftcc_internal.cuh -- handle layout, launch helpers and kernel entry points
// shared by the translation units of libpftcc_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pftcc_b200.h"

namespace pftcc {

// Layout of the data held in HBM (all "K" counts run over kfrom..kto, "Ks" over
// kfrom..kstop):
//   refs_even/odd [nrefs][K][P] float2     (pfts_refs_even/odd(P, kfrom:kto, nrefs))
//   ptcls         [nptcls][K][P] float2    (pfts_ptcls(P, kfrom:kto, nptcls))
//   ctfmats       [nptcls][K][P] float     (ctfmats(P, kfrom:kto, nptcls))
//   polar         [K][2N] float            (polar(2N, kfrom:kto))
//   argtransf     [K][N] double, argtransf1 [N] double
struct Geom {
    int N, P, K, Ks, kfrom, kto, kstop, box;
};

// per-shift phase tables used by the exact kernels: shmat for a list of shifts is
// generated on the device from argtransf in double precision (gen_shmat_8)
// The packed spectrum the stage-2 transform consumes: for the Hermitian contraction
// output X(m), m = 0..P, Z(j) = [X(j) + conj X(P-j)] + i [X(j) - conj X(P-j)] w_N^{-j}
// (j < P; X(0) and X(P) taken as real), whose length-P DFT z(l) = y(2l) + i y(2l+1)
// gives every rotation's correlation sum y(rot) = sum_{m<N} X(m) w_N^{-m rot}.
__device__ __forceinline__ float2 make_z(float2 a, float2 b, float2 wn)   // a = X(j), b = X(P-j)
{
    const float2 E = make_float2(a.x + b.x, a.y - b.y);
    const float ox = a.x - b.x, oy = a.y + b.y;
    const float2 O = make_float2(ox * wn.x - oy * wn.y, ox * wn.y + oy * wn.x);
    return make_float2(E.x - O.y, E.y + O.x);
}

// w_N^{-j} in single precision (FP64 angle, rounded once)
__device__ __forceinline__ float2 wn_of(int j, int N)
{
    double s, c;
    sincospi(-2.0 * j / N, &s, &c);
    return make_float2((float)c, (float)s);
}

struct Work {           // one (reference, shift) correlation for the particle of a group
    int iref;           // 0-based
    int ishift;         // index into the shift list (-1 = no shift, gencorrs_cc_1)
    long long out;      // output offset (MODE_FULL) or candidate id (MODE_BEST)
};

struct Group {          // all work items of one particle slot
    int slot;
    int first, count;   // range in the Work array
    int out_best;       // index of the pftcc_best written in MODE_BEST
};

enum { MODE_FULL = 0, MODE_BEST = 1, MODE_ITEMMAX = 2 };   // ITEMMAX: out[w.out] = max over rotations

// One wave of a tcgen05 stage-1 launch: the (reference, shift) row tiles [rtile0, rtile0 + n_rtiles)
// of the packed row operand against the particle tiles [ptile0, ptile0 + n_ptiles) of the packed
// particle operand (tiles counted from the parity group's first column), into the packed spectrum
// X = Z [P][xcols][xrows] with xrows = 32 n_rtiles, xcols = 128 n_ptiles.  item0: the wave's first
// work item (plane pair, particle tile) in the launch, the prefix over the waves before it.
struct S1Wave {
    float2 *X;
    int rtile0, n_rtiles, ptile0, n_ptiles;
    int item0, xrows, xcols, pad;
};

// One wave of a stage-2 launch: the particle columns [col0, col0 + cols) (absolute column order)
// against the (reference, shift) rows [row0, row0 + rows) of Z = X [P][xcols][xrows]; row row0 + i
// sits at Z row rofs + i, column col0 + c at Z column zc0 + c; the normalising factors D
// [reference - r0][dcols][dlen] hold column col0 + c at c.  blk0: the wave's first block in the
// launch (one block per column).
struct S2Wave {
    const float2 *X;
    const float *D;
    int row0, rows, rofs, xrows, xcols;
    int col0, cols, zc0, r0, dcols;
    int blk0, pad;
};

// state of the tcgen05 stage 1 (packed operand geometry, the device tables of a launch's waves and
// their tensor maps, device error word)
struct UmmaState {
    int Kp = 0, KC = 0, rtiles = 0, ptiles = 0, group_c0 = 0, sms = 0;
    int *err = nullptr;
    S1Wave *d_waves = nullptr;
    void *d_maps = nullptr;     // CUtensorMap[waves_cap], 64-byte aligned
    int waves_cap = 0;
    S2Wave *d_s2waves = nullptr;   // the stage-2 launch's waves
    int s2waves_cap = 0;
};

// m-domain search workspace (sized on first use, reused across calls)
struct SearchWS {
    int nshifts = 0, nrs = 0, nrs_pad = 0, np_pad = 0, M = 0, Mpad = 0;
    int W_rows = 0, W_cols = 0;  // the wave the buffers were sized for
    float2 *UA = nullptr;        // [M][nrs_pad][Ks] ref-side spectra (FP32 path)
    float2 *UB = nullptr;        // [M][np_pad][Ks] particle-side spectra (FP32 path)
    double2 *RU = nullptr;       // [nrefs][J][Ks] spectra of |ref|^2, J = P/2+1
    double2 *CV = nullptr;       // [np_pad][J][Ks] spectra of CTF^2
    float2 *RUf = nullptr;       // [J][Ks][nrefs] FP32 copy of RU for the normaliser's contraction
    float2 *CVf = nullptr;       // [J][Ks][np_pad] FP32 copy of CV
    float *D = nullptr;          // [wave refs][np_pad][P] rotation-dependent normaliser
    float2 *Yn = nullptr;        // [wave refs][wave cols][P/2+1] its spectra (k_norm_y2)
    float2 *X = nullptr;         // [M][wave rows][wave cols] stage-1 output of one wave
    size_t X_elems = 0;
    size_t D_bytes = 0, Y_bytes = 0;   // D and Y capacities of the grouped search (0 otherwise)
    size_t perm_bytes = 0;             // capacity of the grouped search's column order (cand_ref)
    float2 *cand = nullptr;      // [np_pad][8] packed (cc, rs*N+rot) candidates
    float *sqp = nullptr;        // [np_pad]
    __nv_bfloat16 *A16 = nullptr;  // tcgen05 operands, see k_umma.cu
    __nv_bfloat16 *B16 = nullptr;
    size_t A16_elems = 0, B16_elems = 0;
    float *shifts = nullptr;     // [nshifts][2]
    pftcc_best *best = nullptr;  // [np_pad]
    int *cand_ref = nullptr;
    int ptcl_spectra_valid = 0;  // particle spectra current for this handle state
    UmmaState umma;
};

}  // namespace pftcc

struct pftcc_handle {
    pftcc_config cfg{};
    pftcc::Geom g{};
    int nrefs = 0, nptcls = 0;
    int pfrom = 0, pto = 0;
    std::vector<int> pinds;              // global - pfrom -> slot + 1 (0 = not held)
    std::vector<uint8_t> iseven;         // per slot
    int dev = 0;
    cudaStream_t stream = nullptr;
    // device data
    float2 *refs_even = nullptr, *refs_odd = nullptr, *ptcls = nullptr;
    float *sqsums = nullptr, *ctfmats = nullptr;
    uint8_t *d_iseven = nullptr;
    pftcc_ctfparams *d_ctfp = nullptr;
    std::vector<pftcc_ctfparams> h_ctfp;
    int ctf_ready = 0;
    float *polar = nullptr;
    double *argtransf = nullptr, *argtransf1 = nullptr;
    std::vector<float> h_polar;
    std::vector<double> h_argtransf, h_argtransf1;
    std::vector<float> angtab;           // degrees
    // polarizer tables
    int *pol_off = nullptr;
    float *pol_w = nullptr;
    int pol_griddev = -1;
    void *pol_stage = nullptr;           // device staging of host images
    size_t pol_stage_bytes = 0;
    // the volume's expanded FT for polar projection (expand_cmat), side box + 5
    float2 *vol_cube = nullptr;
    int vol_box = 0;
    // matched-filter mode: ref_optlp(kfrom:kstop, nrefs) as [nrefs][Ks] (1 until set_ref_optlp)
    // and the shell factors of shellnorm_and_filter_ref [2 sets][nrefs][Ks]
    float *d_optlp = nullptr;
    float *d_snorm = nullptr;
    int pssnr = 0;                       // params_glob%l_pssnr (within the matched-filter mode)
    // particle ingestion state (k_ingest.cu: cuFFT plans and scratch)
    void *ingest = nullptr;
    // the orientation derivatives of the references (fdf_project_polar), [nrefs][3][K][P]
    float2 *drefs_even = nullptr, *drefs_odd = nullptr;
    // Euclidean objective: cc_objfun, sigma2_noise(kfrom:kto, sig_from:sig_to) as assigned
    // (host copy), its columns in slot order on the device, pixels per shell
    int objfun = PFTCC_OBJFUN_CC;
    std::vector<float> h_sig2;
    int sig_from = 0, sig_to = -1;
    int sig_dirty = 1;
    int sig_uncovered = 0;               // held particles outside sig_from:sig_to
    float *d_sig2 = nullptr;             // [slots][K]
    float *d_pxls = nullptr;             // [K]
    // small per-call device buffers
    pftcc::Work *d_work = nullptr;
    pftcc::Group *d_groups = nullptr;
    size_t work_cap = 0, group_cap = 0;
    float *d_out = nullptr;
    size_t out_cap = 0;
    float *d_shifts = nullptr;
    size_t shifts_cap = 0;
    double *d_dout = nullptr;
    size_t dout_cap = 0;
    pftcc_best *d_best = nullptr;
    size_t best_cap = 0;
    pftcc::SearchWS ws;
    std::mutex mtx;
    std::string last_err;
    long long launches = 0;
    long long wait_limit = 0;            // pipeline-wait polls of the tcgen05 kernels (0 = default)
    pftcc_tuning tune{};                 // wave and tile sizes of the m-domain search (0 = automatic)
    cudaStream_t own_stream = nullptr;
    // pinned host staging of the small per-call tables (column order, shifts, wave tables): one
    // arena for calls made outside stream capture, one for a captured call, whose memcpy nodes
    // read it at every replay
    void *pin[2] = {nullptr, nullptr};
    size_t pin_cap[2] = {0, 0}, pin_off[2] = {0, 0};
    size_t pin_total = 0;    // staging bytes since the last uncaptured grouped search began
    size_t pin_need = 0;     // staging bytes of the last uncaptured grouped search
    // per-kernel-class event timing
    int prof = 0;
    struct ProfEv { int cls; cudaEvent_t a, b; };
    std::vector<ProfEv> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    double prof_ms[PFTCC_K_COUNT] = {};
    long long prof_n[PFTCC_K_COUNT] = {};
};

namespace pftcc {
// records a start event on construction and a stop event on destruction when the
// handle's profiling is on; wrap one kernel launch of class cls
struct KTimer {
    pftcc_handle *h;
    int cls;
    cudaEvent_t a = nullptr, b = nullptr;
    KTimer(pftcc_handle *h_, int cls_);
    ~KTimer();
};
}  // namespace pftcc

namespace pftcc {

// Lets `kernel` use `bytes` of dynamic shared memory: its limit is raised once per device to
// the device's opt-in maximum (less the kernel's static shared memory) -- one fixed value,
// so concurrent callers that launch the kernel with different sizes never lower the limit
// under each other; cudaErrorInvalidValue when `bytes` exceeds it.
cudaError_t smem_limit(const void *kernel, size_t bytes);

int set_err(pftcc_handle *h, int code, const std::string &msg);
int cuda_err(pftcc_handle *h, cudaError_t e, const char *what);
int dev_alloc(pftcc_handle *h, void **p, size_t bytes, const char *what);
void dev_free(pftcc_handle *h, void *p);
int ensure(pftcc_handle *h, void **p, size_t *cap, size_t bytes, const char *what);
// whether the handle's stream is capturing a CUDA graph
bool capturing(const pftcc_handle *h);
// a host table to the device through the pinned staging arena of the call's kind (see the
// handle's pin fields); outside capture the arena wraps (after the stream drains) and grows
int stage_upload(pftcc_handle *h, void *dst_dev, const void *src, size_t bytes, const char *what);

// ---- kernels (launch wrappers return cudaError_t of the launch) ---------------------
cudaError_t launch_polarize(pftcc_handle *h, const float2 *cmats, int n, int first_slot);
cudaError_t launch_expand_cmat(pftcc_handle *h, int box, const float2 *half, float factor, float2 *cube);
cudaError_t launch_fproject_polar(pftcc_handle *h, int box, const float2 *cube, const double *R, const int *mask, int n,
                                  int griddev, float2 *out);
// fdf_project_polar: RD = 36 doubles per reference (R, then dR/de1..3); out [n][K][P],
// dout [n][3][K][P]
cudaError_t launch_fdf_project_polar(pftcc_handle *h, int box, const float2 *cube, const double *RD, int n,
                                     float2 *out, float2 *dout);
cudaError_t launch_ctfmat(pftcc_handle *h, const pftcc_ctfparams *params, int n, float *out, float ddf,
                          int derivative);
cudaError_t launch_sqsums(pftcc_handle *h, int first_slot, int n);
// rotmask (optional) [ngroups][N]: MODE_BEST / MODE_ITEMMAX take their maxima over the
// rotations whose mask byte is non-zero
cudaError_t launch_exact(pftcc_handle *h, const Group *groups, int ngroups, const Work *work,
                         const float *shifts, int mode, int frame, int cc1_kstop, float *out,
                         pftcc_best *best, const uint8_t *rotmask = nullptr);
// single-rotation correlation requests for k_for_rot: iref 0-based, slot, irot 1-based,
// ctf_mode 0 = the stored |CTF| matrices (the drop-in calls), 1 = |CTF| recomputed at
// defocus + ddf; out5 [n][5] = f, df/dsx, df/dsy, df/ddf, unused
struct RotReqH { int iref, slot, irot, ctf_mode; double sx, sy, ddf; };
cudaError_t launch_rot_reqs(pftcc_handle *h, const void *reqs_dev, int n, double *out5);
cudaError_t launch_for_rot(pftcc_handle *h, int iref, int slot, double sx, double sy, int irot,
                           int match_filt, int want_grad, double ddf, double *out5);
cudaError_t launch_grad_batch(pftcc_handle *h, const pftcc_grad_req *req_dev, const int *slots_dev, int nreq,
                              double *out4);
cudaError_t launch_zero_beyond_kstop(pftcc_handle *h);

// k_exact frame of the Euclidean objective: reference frame with shell weights
// pxls(k) / (P sigma2(k)) and the distance's constant terms (gencorrs_euclid_1/_2)
constexpr int FRAME_EUCLID = 2;
inline int exact_frame(const pftcc_handle *h)
{
    return h->objfun == PFTCC_OBJFUN_EUCLID ? FRAME_EUCLID : h->cfg.ctf_frame;
}
// the exact kernel's Euclidean objective is the reference's (reference frame); in the particle
// frame the Euclidean objective is served by the m-domain search alone
int exact_objfun_ok(pftcc_handle *h);
// gencorr_cont_shift_grad_cc_for_rot_8 for nreq requests (k_orisrch.cu; the request layout of
// EuclidReq): out6[nreq][6] = f, d/de1..3, d/dsx, d/dsy
struct EuclidReq;
cudaError_t launch_cont_shift_grad(pftcc_handle *h, const EuclidReq *reqs_dev, int nreq, double *out6);
// particle ingestion (k_ingest.cu): prepimg4align of n <= cap images [n][B][B] into cap half-plane
// FTs [cap][box][box/2+1] (box = boxmatch); xy [n][2], flag [n], ctf [n] on the device
int ingest_images(pftcc_handle *h, const float *imgs_dev, int n, int cap, int B, const float *xy_dev,
                  const int *flag_dev, const pftcc_ctfparams *ctf_dev, const pftcc_prep_opts &opts, float2 *cm_out);
int ingest_batch_max(int B);
void ingest_free(pftcc_handle *h);
// euler2m (and with dR, euler2dm per radian) of Spider angles in degrees, row-major, FP64
void host_euler2m(const double e[3], double *R, double *dR);
// batched pftcc_orisrch_grad%minimize (k_orisrch.cu); the caller holds the lock
int orisrch_batch(pftcc_handle *h, int n, const pftcc_orisrch_req *req, int maxits, double pgtol, double factr,
                  pftcc_orisrch_out *out);
// calc_ptcl_pspec: mean power per shell of slot's particle, all K shells, into pspec_dev[K]
cudaError_t launch_ptcl_pspec(pftcc_handle *h, int slot, float *pspec_dev);
// matched-filter mode (k_matchfilt.cu): the shell factors of references r0..r0+n-1 (both sets);
// the factors of reference set `set` on the m-domain spectra; prep_matchfilt requests
// {iref (0-based), slot, irot, pad}
cudaError_t launch_shellnorm(pftcc_handle *h, int r0, int n);
cudaError_t launch_shellnorm_apply(pftcc_handle *h, int M, int nrs, int rows_pad, int nshifts, int set, float2 *UA,
                                   double2 *RU);
cudaError_t launch_prep_matchfilt(pftcc_handle *h, const void *reqs_dev, int nreq);
// allocates ref_optlp (ones) and the factors on first use and computes the factors of references
// r0..r0+n-1 when match_filt is on; snorm_ptr(h) is the factor array or null when it is off
int snorm_ready(pftcc_handle *h, int r0, int n);
inline const float *snorm_ptr(const pftcc_handle *h) { return h->cfg.match_filt ? h->d_snorm : nullptr; }
// sigma2_noise on the device and covering every held particle (rebuilt first when stale
// and may_alloc); PFTCC_OK or the error code, with the message set
int euclid_ready(pftcc_handle *h, int may_alloc);
// one single-rotation Euclidean request (k_euclid.cu); iref 0-based, slot = particle slot
struct EuclidReq { int iref, slot, irot, pad; double sx, sy; };
// out3[nreq][3] = f, df/dsx, df/dsy (with_f); shells[nreq][3][K] = sigma_contrib,
// ptcl_sumsq, ref_sumsq over every shell (want_shells)
cudaError_t launch_euclid_rot(pftcc_handle *h, const EuclidReq *reqs_dev, int nreq, int with_f, int want_shells,
                              double *out3, double *shells);

// adjoint requests served in one launch (pftcc_capi.cu; caller holds the handle lock)
int grad_batch_host(pftcc_handle *h, int nreq, const pftcc_grad_req *req, double *f, double *grad3);
// one genfrc / specscore request (reference frame); iref 0-based, slot = particle slot
struct FrcReq { int iref, slot, irot, has_shift; double sx, sy; };
cudaError_t launch_specscore(pftcc_handle *h, const FrcReq *reqs_dev, int nreq, float *frc_dev, float *score_dev);
// batched bound-constrained quasi-Newton refinement (refine.cu)
int refine_batch(pftcc_handle *h, int n, const pftcc_refine_req *req, const double *lb, const double *ub, int maxits,
                 double pgtol, double factr, pftcc_refine_out *out);

// batched pftcc_shsrch_grad (shsrch.cu); slots[n] the particles' slots, the caller holds the lock
int shsrch_batch(pftcc_handle *h, int mode, const pftcc_shsrch_opts &o, int n, const pftcc_shsrch_req *req,
                 const int *slots, pftcc_shsrch_out *out);

// tcgen05 stage 1 (k_umma.cu): every wave of the list in one persistent launch (the waves' X,
// rtile0, n_rtiles, ptile0, n_ptiles given; item0, xrows and xcols filled in), after the operands
// were packed by umma_stage1(..., prepare = 1, ...)
int umma_stage1_waves(pftcc_handle *h, int M, std::vector<S1Wave> &waves);
// the device error word cleared once per search (every stage-1 launch of the search may set it)
int umma_reset(pftcc_handle *h);
int umma_check(pftcc_handle *h);
void umma_free(pftcc_handle *h);

// m-domain search (k_search.cu)
int search_mdomain(pftcc_handle *h, int nshifts, const float *shifts_host, int precision, int ntop,
                   pftcc_best *out_dev, float *ccall_dev);
// the grouped search: group q's particle slots [slot0[q], +nslot[q]) against its references
// [ref0[q], +nref[q]) (0-based), every group's waves in shared launches
int search_mdomain_groups(pftcc_handle *h, int ngroups, const int *ref0, const int *nref, const int *slot0,
                          const int *nslot, int nshifts_in, const float *shifts_host, int precision, int ntop,
                          pftcc_best *out_dev, int check);

}  // namespace pftcc

#define PFTCC_LAUNCH(h) (++(h)->launches)

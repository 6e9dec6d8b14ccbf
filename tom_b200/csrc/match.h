// FLCF matching plan (see match.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "ctx.h"

namespace tg {

bool match_sizes_supported(const int N[3], const int T[3]);

// the stages on the run-time line engine for edges without compiled kernels
// (match_rt.cu); the c2r kernels take the x edge itself, which may be odd
bool match_rt_length_ok(int L);
cudaError_t launch_spec_x_rt(int NX, const float* t2, const float* mask, float2* A, const int T[3], int d0x, int nb,
                             double* tsum, cudaStream_t st);
cudaError_t launch_spec_z_rt(int NZ, const float2* A, float2* Z, const int T[3], int d0z, int nh1, int nb,
                             cudaStream_t st);
cudaError_t launch_corr_y_rt(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                             long long ncols, int nb, cudaStream_t st);
cudaError_t launch_inv_z_rt(int NZ, const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st);
cudaError_t launch_c2r_flcf_rt(int NX, const float2* H, const float* mu0, const float* gam, const double* tsum,
                               int Ny, int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                               float* maxcc, int* angidx, cudaStream_t st);
cudaError_t launch_c2r_map_rt(int NX, const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                              int Nz, float inv_nm, double c, double inv_m, double mu_t, float* cc, cudaStream_t st);

// register-resident hot kernels (match_fast.cu) for the sizes they cover
bool fast_corr_y(int NY, int Ty);
bool fast_inv_z(int NZ);
bool fast_c2r(int NH);
bool fast_spec_z(int NZ, int Tz);
cudaError_t launch_spec_z_fast(int NZ, const float2* A, float2* Z, int Ty, int Tz, int d0z, int nh1, int nb,
                               cudaStream_t st);
// tmem: the y edge 512's columns keep F_I and their twiddles in tensor memory
cudaError_t launch_corr_y_fast(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                               long long ncols, int nb, cudaStream_t st, bool tmem = false);
cudaError_t launch_inv_z_fast(int NZ, const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st);
cudaError_t launch_c2r_fast(int NH, const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                            int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                            float* maxcc, int* angidx, cudaStream_t st);
// the 928 / 464 edges (match_fast29.cu)
cudaError_t launch_corr_y_p928(const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y, long long ncols,
                               int nb, cudaStream_t st);
cudaError_t launch_inv_z_p464(const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st);
cudaError_t launch_c2r_p464(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st);
// the 128 edges (match_fast128.cu)
cudaError_t launch_inv_z_b128(const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st);
cudaError_t launch_c2r_h256(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st);
cudaError_t launch_c2r_b128(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st);
cudaError_t launch_c2r_b64(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                           int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                           int* angidx, cudaStream_t st);
// x edge 512 with TMA tile loads (match_tma.cu); err: the context's device error word
bool tma_c2r_available();
cudaError_t launch_c2r_t256(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, int* err, cudaStream_t st);
// x edge 928 with TMA tile loads (match_fast29.cu)
cudaError_t launch_c2r_t464(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, int* err, cudaStream_t st);
// z edge 256 with the radix-16 stages on tcgen05 tensor cores (inv_z_tc.cu)
cudaError_t launch_inv_z_tc256(const float2* Q, float2* H, int Ny, int nh1, int nb, int* err, cudaStream_t st);
cudaError_t c2c3d_batch(float2* data, const int t[3], int nb, int dir, double scale, cudaStream_t st);
cudaError_t c2c3d_batch64(double2* data, const int t[3], int nb, int dir, double scale, cudaStream_t st);

struct PeakAnalysis;

struct MatchPlan {
    tomgpu_ctx* ctx = nullptr;
    int N[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    int B = 8;
    bool generic_only = false;  // force the generic kernels (tests compare both paths)
    bool no_tma = false;        // the cp.async x-line kernel for the 512 x edge (comparisons)
    bool tc_inv_z = false;      // the z edge 256's inverse z-DFT on tcgen05 tensor cores
    long long nvox = 0, nh1 = 0, tn = 0;
    int64_t bytes_held = 0;
    int64_t batch_bytes = 0;
    bool has_template = false, has_volume = false, has_psf = false;
    std::vector<float> h_mask;  // host copy of the mask the volume statistics were made with
    double msize = 0, tmean = 0, tstd = 0, vmean = 0;
    // template state
    float* d_tmpl = nullptr;  // tom_norm'ed template
    float* d_mask = nullptr;
    float* d_wu = nullptr;    // ifftshift(psf): weight in unshifted frequency order
    // volume state
    float2* d_fimg = nullptr;  // spectrum of I - c, [kx][kz][ky]
    float* d_mu0 = nullptr;    // local mean of I - c
    float* d_sig = nullptr;    // local std
    float* d_gam = nullptr;    // 1 / (sigma_T sigma_I) or 0
    // per-batch work
    float* d_mats = nullptr;
    float* h_mats = nullptr;
    int mats_cap = 0;
    cudaEvent_t ev_mats = nullptr;
    float* d_t1 = nullptr;
    float2* d_tc = nullptr;
    double* d_tsum = nullptr;
    float2* d_A = nullptr;
    float2* d_Z = nullptr;
    float2* d_Q = nullptr;
    float2* d_H = nullptr;
    double* d_tmp64 = nullptr;
    // per-rotation peak analysis (PSR / autocorrelation maps), created on first use
    PeakAnalysis* an = nullptr;
    float *d_cc = nullptr, *d_psr = nullptr, *d_soc = nullptr, *d_auto = nullptr;

    ~MatchPlan();
    void release();
    int alloc(void** p, size_t bytes);
    int create(tomgpu_ctx* c, const int vol[3], const int tm[3], int batch, bool generic);
    int alloc_batch(int nb);
    int64_t batch_need(int nb) const;  // bytes alloc_batch(nb) allocates
    int default_batch() const;
    int check_ready();
    void free_batch();
    int autotune(const float* eulers, int R, const int* cands, int nc, int* best, float* ms_per_rot);
    int ensure_mats(int R);
    int upload_mats(const float* eulers, int R);
    // raw: take the template as given (tom_os3_corr's own statistics) instead
    // of findTemplate's tom_norm and filter
    int set_template(const float* tmpl, const float* mask, const float* psf, bool raw = false);
    int set_volume(const float* vol);
    int prepare_batch(int off, int nb);
    int run(const float* eulers, int R, int index_offset, float* maxcc, int* angidx);
    int corr(const float* t, float* cc);
    int cc_map_tail(float* cc);  // corr_y, inv_z and the FLCF map of the prepared rotation
    int run_analysis(const float* eulers, int R, int index_offset, int flags, float* maxcc, int* angidx,
                     float* psr, float* soc);
    int init_results(float* maxcc, int* angidx);
    int rescore(const float* vol, const float* eulers, const int* pos1, int K, double* out);
};

int corr_norm(tomgpu_ctx* ctx, const float* a, const float* b, const int n[3], const float* mask, const float* psf1,
              const float* psf2, float* out);
// scratch: workspace reused across jobs (align_scratch_new), or NULL for a private one
struct AlignScratch;
AlignScratch* align_scratch_new();
void align_scratch_free(AlignScratch* s);
// Buffer i of the scratch's pool, grown to at least bytes (contents not kept);
// nullptr when the allocation fails.
void* align_scratch_buffer(AlignScratch* s, int i, size_t bytes);
int align_job(tomgpu_ctx* ctx, const tomgpu_align_job& job, float angles_out[3], float shifts_out[3],
              float* peak_out, size_t budget_voxels, AlignScratch* scratch);
// tom_angles2rotmatrix of (phi, psi, theta) in degrees, column-major, rounded to float
void rotmatrix_as_float(double phi, double psi, double theta, float m9[9]);
// the values of an angle range [start increment end] (one value when increment = 0)
std::vector<double> axis_values(const float r[3]);
// the step after a job's scan: angle of the first maximum of cmax * mask_ccf,
// one more tom_corr at that angle, spline peak; nph / nps the phi and psi
// counts; all work on stream st, which it synchronises
int align_finish(tomgpu_ctx* ctx, cudaStream_t st, const tomgpu_align_job& job, int nph, int nps,
                 const float* cmax, const float* amax, double nmask, AlignScratch* sc, float angles_out[3],
                 float shifts_out[3], float* peak_out);
// The fused alignment engine (align_fused.cu): jobs of one cubic box edge it
// compiles, all with or all without wedges, scanned as one batch of
// (particle, rotation) entries.  job_idx lists the jobs; outputs are indexed
// by job.  budget_bytes bounds the per-batch spectra (0: the default);
// allow_prune lets the last inverse DFT run only where mask_ccf is non-zero.
bool align_fused_supported(const tomgpu_align_job& job);
int align_fused(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, const int* job_idx, int n, float* angles,
                float* shifts, float* peaks, size_t budget_bytes, bool allow_prune, AlignScratch* sc);
int av3_average_add(tomgpu_ctx* ctx, const int n[3], const tomgpu_avg_item* items, int K, double* avg, double* wei);
int corr3d_peaks(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt, const float* const* particles,
                 int np, const double* angles_deg, int nang, const float* mask, const tomgpu_wedge_spec* wedge_t,
                 const tomgpu_wedge_spec* wedge_p, const float* mask_cc, double* peak, double* val, int32_t* angle_idx);
int av3_average_final(tomgpu_ctx* ctx, const int n[3], const double* avg, const double* wei, double* out);

}  // namespace tg

struct tomgpu_match_plan {
    tg::MatchPlan p;
};

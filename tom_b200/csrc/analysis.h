// Peak analysis of FLCF maps: PSR and autocorrelation (SOC) maps (see analysis.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "ctx.h"

namespace tg {

// tom_os3_sphereMask of a box of size T (radius floor(T/2)-1 around floor(T/2);
// a non-cubic box gives ones).
void os3_sphere_mask_host(const int T[3], std::vector<float>& m);

// State for the peak analysis of maps of size N found with templates of size
// T: the FP64 spectra of the PSR and correlation-mask convolution kernels and
// the work buffers (about 5 half spectra and 3 real volumes in FP64).
struct PeakAnalysis {
    tomgpu_ctx* ctx = nullptr;
    int N[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    long long nvox = 0, hs = 0, tn = 0;
    double m_psr = 0, m_msk = 0, m_sph = 0;  // nonzero counts of the masks
    double2 *f_psr = nullptr, *f_msk = nullptr, *f1 = nullptr, *f2 = nullptr, *f3 = nullptr;
    double *v64 = nullptr, *m1 = nullptr, *m2 = nullptr;
    float *mu = nullptr, *sig = nullptr, *gam = nullptr;
    float *d_mask = nullptr, *d_sph = nullptr, *d_am = nullptr, *d_psrbox = nullptr, *tmp_t = nullptr;
    double2 *z = nullptr, *zs = nullptr;
    double *acsd = nullptr, *sc = nullptr;

    ~PeakAnalysis();
    void release();
    int alloc(void** p, size_t bytes);
    // mask_dev: the correlation mask (template-sized); NULL = tom_os3_sphereMask
    int create(tomgpu_ctx* c, const int vol[3], const int tm[3], const float* mask_dev);
    // A = tom_os3_corr(t, t) (template-sized)
    int autocorr(const float* t, float* A);
    // spectra of the peak map and its square; precede psr and soc
    int spectra(const float* pk);
    int local_moments(const double2* fk, double msize);
    int psr(const float* pk, float* out);
    int soc(const float* pk, const float* A, float* out);
};

int analysis_update(tomgpu_ctx* ctx, const float* cc, const float* psr, const float* soc, long long n, int flags,
                    int index, float* o_cc, int* o_idx, float* o_psr, float* o_soc);
int analysis_init(tomgpu_ctx* ctx, long long n, float* o_cc, int* o_idx, float* o_psr, float* o_soc);

}  // namespace tg

#pragma once
#include <cuda_runtime.h>
namespace tg {
cudaError_t weight3d(float* w, const int dims[3], const float* d_fx, const float* d_fy, const float* d_fz,
                     const float* d_nrm, int n_tilt, cudaStream_t st);
cudaError_t wedge(float* out, const int dims[3], double t1, double t2, int av3, cudaStream_t st);
cudaError_t ifftshift_real(const float* in, float* out, const int dims[3], cudaStream_t st);
// FP64 sums (result written to the device double *out)
cudaError_t sum_affine_f32(const float* a, long long n, double s, double o, double* out, cudaStream_t st);
cudaError_t sum_sqdev_f32(const float* a, long long n, double s, double o, double mean, double* out, cudaStream_t st);
cudaError_t sum_f64(const double* a, long long n, double* out, cudaStream_t st);
cudaError_t count_nonzero(const float* a, long long n, double* out, cudaStream_t st);
cudaError_t norm_under_mask_sums(const double* v, const float* m, long long n, double* d_mean_num,
                                 double* d_var_num, double mea, int which, cudaStream_t st);
// elementwise
cudaError_t affine_f32_to_f64(const float* a, double* b, long long n, double s, double o, cudaStream_t st);
cudaError_t normalize_f32(const float* a, float* b, long long n, double s, double o, double m, double inv,
                          cudaStream_t st);
cudaError_t square_f64(double* a, long long n, cudaStream_t st);
cudaError_t mul_c64(double2* a, const double2* b, long long n, cudaStream_t st);
cudaError_t real_to_c64(const float* a, double2* b, long long n, cudaStream_t st);
cudaError_t mul_weight_c64(double2* a, const float* w, long long n, cudaStream_t st);
cudaError_t re_c64(const double2* a, double* b, long long n, double s, cudaStream_t st);
cudaError_t double_to_float(const double* a, float* b, long long n, cudaStream_t st);
cudaError_t stats_final(const double* m1, const double* m2, float* mu, float* sig, long long n, cudaStream_t st);
cudaError_t gamma_from_sigma(const float* sig, float* gam, long long n, double tstd, cudaStream_t st);
cudaError_t place_f64(const float* small, const int t[3], double* big, const int nn[3], const int off[3],
                      cudaStream_t st);
}  // namespace tg

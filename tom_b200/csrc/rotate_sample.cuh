// rot3d's per-voxel sampling (Sptrans/tom_rotatec.c:291-399) as an inline
// device function, shared by the rotation and alignment kernels.  Explicit
// round-to-nearest intrinsics keep the float operation order of the
// reference, so results are bit-identical to rot3d.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace tg {

__device__ __forceinline__ float rot_sample(const float* __restrict__ in, int sx, int sy, int sz,
                                            const float* m, float px, float py, float pz, int i,
                                            int j, int k) {
    const float di = (float)(long long)__fsub_rn((float)i, px);
    const float dj = (float)(long long)__fsub_rn((float)j, py);
    const float dk = (float)(long long)__fsub_rn((float)k, pz);
    const float rx = __fadd_rn(__fadd_rn(__fadd_rn(px, __fmul_rn(m[0], di)), __fmul_rn(m[1], dj)),
                               __fmul_rn(m[2], dk));
    if (rx < 0.f || rx > (float)(sx - 1)) return 0.f;
    const float ry = __fadd_rn(__fadd_rn(__fadd_rn(py, __fmul_rn(m[3], di)), __fmul_rn(m[4], dj)),
                               __fmul_rn(m[5], dk));
    if (ry < 0.f || ry > (float)(sy - 1)) return 0.f;
    const float rz = __fadd_rn(__fadd_rn(__fadd_rn(pz, __fmul_rn(m[6], di)), __fmul_rn(m[7], dj)),
                               __fmul_rn(m[8], dk));
    if (rz < 0.f || rz > (float)(sz - 1)) return 0.f;
    const int fx = (int)rx, fy = (int)ry, fz = (int)rz;
    const float wx = __fsub_rn(rx, (float)fx), wy = __fsub_rn(ry, (float)fy), wz = __fsub_rn(rz, (float)fz);
    const float ux = __fsub_rn(1.f, wx), uy = __fsub_rn(1.f, wy), uz = __fsub_rn(1.f, wz);
    const long long sxy = (long long)sx * sy;
    const long long b = fx + (long long)fy * sx + (long long)fz * sxy;
    const bool ex = fx == sx - 1, ey = fy == sy - 1, ez = fz == sz - 1;
    const float v000 = __ldg(in + b);
    const float v100 = ex ? 0.f : __ldg(in + b + 1);
    const float v010 = ey ? 0.f : __ldg(in + b + sx);
    const float v110 = (ex || ey) ? 0.f : __ldg(in + b + sx + 1);
    const float v001 = ez ? 0.f : __ldg(in + b + sxy);
    const float v101 = (ex || ez) ? 0.f : __ldg(in + b + sxy + 1);
    const float v011 = (ey || ez) ? 0.f : __ldg(in + b + sxy + sx);
    const float v111 = (ex || ey || ez) ? 0.f : __ldg(in + b + sxy + sx + 1);
    const float a = __fadd_rn(v000, __fmul_rn(__fsub_rn(v100, v000), wx));
    const float bb = __fadd_rn(__fmul_rn(v010, ux), __fmul_rn(v110, wx));
    const float c = __fadd_rn(__fmul_rn(v001, ux), __fmul_rn(v101, wx));
    const float d = __fadd_rn(__fmul_rn(v011, ux), __fmul_rn(v111, wx));
    const float lo = __fadd_rn(__fmul_rn(a, uy), __fmul_rn(bb, wy));
    const float hi = __fadd_rn(__fmul_rn(c, uy), __fmul_rn(d, wy));
    return __fadd_rn(__fmul_rn(lo, uz), __fmul_rn(hi, wz));
}


// The eight corner values of voxel (i, j, k) for rot_sample, as they are
// read there (zero where a corner lies beyond the last voxel of an axis):
// v000 v100 v010 v110 in .x .y .z .w of b[2 v], v001 v101 v011 v111 of b[2 v + 1].
__device__ __forceinline__ void brick_values(const float* __restrict__ in, int sx, int sy, int sz, int i, int j,
                                             int k, float4& lo, float4& hi) {
    const long long sxy = (long long)sx * sy;
    const long long v = i + (long long)j * sx + (long long)k * sxy;
    const bool ex = i == sx - 1, ey = j == sy - 1, ez = k == sz - 1;
    lo.x = in[v];
    lo.y = ex ? 0.f : in[v + 1];
    lo.z = ey ? 0.f : in[v + sx];
    lo.w = (ex || ey) ? 0.f : in[v + sx + 1];
    hi.x = ez ? 0.f : in[v + sxy];
    hi.y = (ex || ez) ? 0.f : in[v + sxy + 1];
    hi.z = (ey || ez) ? 0.f : in[v + sxy + sx];
    hi.w = (ex || ey || ez) ? 0.f : in[v + sxy + sx + 1];
}
__device__ __forceinline__ void brick_corners(const float* __restrict__ in, int sx, int sy, int sz, int i, int j,
                                              int k, float4* __restrict__ b) {
    const long long v = i + (long long)j * sx + (long long)k * sx * sy;
    float4 lo, hi;
    brick_values(in, sx, sy, sz, i, j, k, lo, hi);
    b[2 * v] = lo;
    b[2 * v + 1] = hi;
}

// Corner loads of a brick volume: float bricks (two float4 per voxel) or
// half bricks (one uint4 of eight halves per voxel, for volumes whose values
// are all exact in half precision: the conversion back to float is exact).
__device__ __forceinline__ void brick_load(const float4* __restrict__ bk, int b, float4& lo, float4& hi) {
    lo = __ldg(bk + 2 * b);
    hi = __ldg(bk + 2 * b + 1);
}
__device__ __forceinline__ void brick_load(const uint4* __restrict__ bk, int b, float4& lo, float4& hi) {
    const uint4 u = __ldg(bk + b);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 c = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    const float2 d = __half22float2(*reinterpret_cast<const __half2*>(&u.z));
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&u.w));
    lo = make_float4(a.x, a.y, c.x, c.y);
    hi = make_float4(d.x, d.y, f.x, f.y);
}

// rot_sample reading the corners from a brick volume (brick_corners): the
// same coordinates, bounds and float operations, so the same result, from two
// 16-byte loads (one for half bricks) instead of eight scattered 4-byte ones.
// For integer-valued centres below 2^24 only (i - p is then an exact integer,
// so rot_sample's truncation of it is the identity) and volumes of fewer
// than 2^31 voxels (32-bit brick index).
template <typename BK>
__device__ __forceinline__ float rot_sample_brick(const BK* __restrict__ bk, int sx, int sy, int sz,
                                                  const float* m, float px, float py, float pz, int i, int j,
                                                  int k) {
    const float di = __fsub_rn((float)i, px);
    const float dj = __fsub_rn((float)j, py);
    const float dk = __fsub_rn((float)k, pz);
    const float rx = __fadd_rn(__fadd_rn(__fadd_rn(px, __fmul_rn(m[0], di)), __fmul_rn(m[1], dj)),
                               __fmul_rn(m[2], dk));
    if (rx < 0.f || rx > (float)(sx - 1)) return 0.f;
    const float ry = __fadd_rn(__fadd_rn(__fadd_rn(py, __fmul_rn(m[3], di)), __fmul_rn(m[4], dj)),
                               __fmul_rn(m[5], dk));
    if (ry < 0.f || ry > (float)(sy - 1)) return 0.f;
    const float rz = __fadd_rn(__fadd_rn(__fadd_rn(pz, __fmul_rn(m[6], di)), __fmul_rn(m[7], dj)),
                               __fmul_rn(m[8], dk));
    if (rz < 0.f || rz > (float)(sz - 1)) return 0.f;
    const int fx = (int)rx, fy = (int)ry, fz = (int)rz;
    const float wx = __fsub_rn(rx, (float)fx), wy = __fsub_rn(ry, (float)fy), wz = __fsub_rn(rz, (float)fz);
    const float ux = __fsub_rn(1.f, wx), uy = __fsub_rn(1.f, wy), uz = __fsub_rn(1.f, wz);
    const int b = fx + sx * (fy + sy * fz);
    float4 lo, hi;
    brick_load(bk, b, lo, hi);
    const float a = __fadd_rn(lo.x, __fmul_rn(__fsub_rn(lo.y, lo.x), wx));
    const float bb = __fadd_rn(__fmul_rn(lo.z, ux), __fmul_rn(lo.w, wx));
    const float c = __fadd_rn(__fmul_rn(hi.x, ux), __fmul_rn(hi.y, wx));
    const float d = __fadd_rn(__fmul_rn(hi.z, ux), __fmul_rn(hi.w, wx));
    const float l2 = __fadd_rn(__fmul_rn(a, uy), __fmul_rn(bb, wy));
    const float h2 = __fadd_rn(__fmul_rn(c, uy), __fmul_rn(d, wy));
    return __fadd_rn(__fmul_rn(l2, uz), __fmul_rn(h2, wz));
}

}  // namespace tg

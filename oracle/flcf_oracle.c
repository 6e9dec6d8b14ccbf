/* CPU restatement of TOM's rotation, peak and weighting routines.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  Nothing in tom_b200/ links or calls it.
 *
 * Every routine restates a reference routine with the same float arithmetic
 * order (no FMA contraction: compile with -ffp-contract=off or plain -O2 on
 * x86-64), so its results equal the reference's bit for bit:
 *
 *   oracle_euler_matrix  Sptrans/tom_rotatec.c:164-288 (exact sin/cos table
 *                        for multiples of 30/45 degrees, ZXZ matrix)
 *   oracle_rot3d         Sptrans/tom_rotatec.c:291-399 (pull mapping with the
 *                        transposed matrix, trilinear, zero outside)
 *   oracle_find_max      Analysis/tom_peakinc.c:23-52 (first strict maximum
 *                        in x-fastest order, start value -99999)
 *   oracle_weight3d      Filtrans/tom_calc_weight_functioninc.c:152-252
 *                        (Radermacher exact weighting)
 */
#include <math.h>
#include <stdint.h>

#define ORACLE_PI 3.14159265358979323846264338327950288

/* cos/sin of angles the reference tabulates exactly (degrees). */
static int exact_trig(float deg, float *c, float *s)
{
    static const float tab_deg[16] = {0, 30, 45, 60, 90, 120, 135, 150,
                                      180, 210, 225, 240, 270, 300, 315, 330};
    const double h3 = sqrt(3.0) / 2.0, h2 = sqrt(2.0) / 2.0;
    const double cs[16] = {1, h3, h2, 0.5, 0, -0.5, -h2, -h3,
                           -1, -h3, -h2, -0.5, 0, 0.5, h2, h3};
    const double sn[16] = {0, 0.5, h2, h3, 1, h3, h2, 0.5,
                           0, -0.5, -h2, -h3, -1, -h3, -h2, -0.5};
    int hit = 0;
    for (int i = 0; i < 16; ++i)
        if (tab_deg[i] == deg) { *c = (float)cs[i]; *s = (float)sn[i]; hit = 1; }
    return hit;
}

static void trig_deg(float deg, float *c, float *s)
{
    if (exact_trig(deg, c, s)) return;
    float rad = (float)(deg * ORACLE_PI / 180.0);
    *c = (float)cos(rad);
    *s = (float)sin(rad);
}

/* m[0..8] = rm00, rm10, rm20, rm01, rm11, rm21, rm02, rm12, rm22 */
void oracle_euler_matrix(const float euler_deg[3], float m[9])
{
    float cphi, sphi, cpsi, spsi, cth, sth;
    trig_deg(euler_deg[0], &cphi, &sphi);
    trig_deg(euler_deg[1], &cpsi, &spsi);
    trig_deg(euler_deg[2], &cth, &sth);
    m[0] = cpsi * cphi - cth * spsi * sphi;
    m[1] = spsi * cphi + cth * cpsi * sphi;
    m[2] = sth * sphi;
    m[3] = -cpsi * sphi - cth * spsi * cphi;
    m[4] = -spsi * sphi + cth * cpsi * cphi;
    m[5] = sth * cphi;
    m[6] = sth * spsi;
    m[7] = -sth * cpsi;
    m[8] = cth;
}

void oracle_rot3d(const float *in, float *out, long sx, long sy, long sz,
                  const float m[9], float px, float py, float pz)
{
    const long sxy = sx * sy;
    const float xmax = (float)(sx - 1), ymax = (float)(sy - 1), zmax = (float)(sz - 1);
    long o = 0;
    for (long k = 0; k < sz; ++k)
        for (long j = 0; j < sy; ++j)
            for (long i = 0; i < sx; ++i, ++o) {
                const float di = (float)(long)(i - px);
                const float dj = (float)(long)(j - py);
                const float dk = (float)(long)(k - pz);
                float rx = px + m[0] * di + m[1] * dj + m[2] * dk;
                if (rx < 0 || rx > xmax) { out[o] = 0; continue; }
                float ry = py + m[3] * di + m[4] * dj + m[5] * dk;
                if (ry < 0 || ry > ymax) { out[o] = 0; continue; }
                float rz = pz + m[6] * di + m[7] * dj + m[8] * dk;
                if (rz < 0 || rz > zmax) { out[o] = 0; continue; }
                const long fx = (long)rx, fy = (long)ry, fz = (long)rz;
                const float wx = rx - fx, wy = ry - fy, wz = rz - fz;
                const float ux = 1 - wx, uy = 1 - wy, uz = 1 - wz;
                const long b = fx + fy * sx + fz * sxy;
                const int ex = fx == sx - 1, ey = fy == sy - 1, ez = fz == sz - 1;
                const float v000 = in[b];
                const float v100 = ex ? 0.f : in[b + 1];
                const float v010 = ey ? 0.f : in[b + sx];
                const float v110 = (ex || ey) ? 0.f : in[b + sx + 1];
                const float v001 = ez ? 0.f : in[b + sxy];
                const float v101 = (ex || ez) ? 0.f : in[b + sxy + 1];
                const float v011 = (ey || ez) ? 0.f : in[b + sxy + sx];
                const float v111 = (ex || ey || ez) ? 0.f : in[b + sxy + sx + 1];
                const float a = v000 + (v100 - v000) * wx;
                const float bb = v010 * ux + v110 * wx;
                const float c = v001 * ux + v101 * wx;
                const float d = v011 * ux + v111 * wx;
                out[o] = (a * uy + bb * wy) * uz + (c * uy + d * wy) * wz;
            }
}

/* R rotations of one volume; eulers R x 3 degrees (phi, psi, theta). */
void oracle_rot3d_batch(const float *in, float *out, long sx, long sy, long sz,
                        const float *eulers, int R, float px, float py, float pz)
{
    const long n = sx * sy * sz;
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < R; ++r) {
        float m[9];
        oracle_euler_matrix(eulers + 3 * r, m);
        oracle_rot3d(in, out + (long)r * n, sx, sy, sz, m, px, py, pz);
    }
}

void oracle_find_max(const float *v, const int dims[3], float *val, int pos[3])
{
    float best = -99999.0f;
    long idx = 0;
    for (int k = 0; k < dims[2]; ++k)
        for (int j = 0; j < dims[1]; ++j)
            for (int i = 0; i < dims[0]; ++i, ++idx)
                if (v[idx] > best) { best = v[idx]; pos[0] = i; pos[1] = j; pos[2] = k; }
    *val = best;
}

/* Frequency coordinate of index i (1-based loop counter semantics of the
 * reference: steps of 1/n that flip sign after the n/2-th sample). */
void oracle_weight3d(float *w, const int dims[3], const double *angles, int n_tilt,
                     double thickness)
{
    const float pi_c = 3.1416f, width = 3.1416f;
    const int thick = (int)thickness;
    float nrm[64][3];
    if (n_tilt > 64) return;
    for (int t = 0; t < n_tilt; ++t) {
        float phi = (float)angles[2 * t] * pi_c / 180;
        float th = (float)angles[2 * t + 1] * pi_c / 180;
        float zw = (float)sin(th) * pi_c * thick;
        nrm[t][0] = (float)zw * (float)cos(phi);
        nrm[t][1] = (float)zw * (float)sin(phi);
        nrm[t][2] = (float)cos(th) * pi_c * thick;
    }
    long o = 0;
    float fz = 0;
    for (int iz = 1; iz <= dims[2]; ++iz) {
        float fy = 0;
        for (int iy = 1; iy <= dims[1]; ++iy) {
            float fx = 0;
            for (int ix = 1; ix <= dims[0]; ++ix) {
                float sum = 0;
                for (int t = 0; t < n_tilt; ++t) {
                    float arg = fx * nrm[t][0] + fy * nrm[t][1] + fz * nrm[t][2];
                    float add;
                    if (fabs(arg) < (float)1e-6) add = 1;
                    else if (fabs(arg) > 1e-6 && fabs(arg) < width) add = (float)sin(arg) / arg;
                    else add = 0;
                    sum = sum + add;
                }
                w[o++] = sum > 1.0 ? (float)(1.0 / sum) : 1.0f;
                fx = fx + (float)1.0 / dims[0];
                if (ix == dims[0] / 2) fx = -fx;
            }
            fy = fy + (float)1.0 / dims[1];
            if (iy == dims[1] / 2) fy = -fy;
        }
        fz = fz + (float)1.0 / dims[2];
        if (iz == dims[2] / 2) fz = -fz;
    }
}

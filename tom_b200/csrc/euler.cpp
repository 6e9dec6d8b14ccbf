// ZXZ rotation matrix exactly as tom_rotatec computes it
// (Sptrans/tom_rotatec.c:164-288): angles equal to a multiple of 30 or 45
// degrees take tabulated cos/sin values (double constants rounded to float),
// all others cos/sin in double of the float radian value; the matrix products
// are float.  Built with -ffp-contract=off so the host arithmetic matches the
// reference bit for bit; the CUDA kernels receive these 9 floats.
#include <cmath>

#include "ctx.h"

namespace tg {

namespace {
bool tabulated(float deg, float* c, float* s) {
    // angle -> (cos, sin) for the angles the reference special-cases
    struct Entry { float deg; double c, s; };
    const double r3 = std::sqrt(3.0) / 2, r2 = std::sqrt(2.0) / 2;
    const Entry table[16] = {
        {0, 1, 0},        {30, r3, 0.5},    {45, r2, r2},      {60, 0.5, r3},
        {90, 0, 1},       {120, -0.5, r3},  {135, -r2, r2},    {150, -r3, 0.5},
        {180, -1, 0},     {210, -r3, -0.5}, {225, -r2, -r2},   {240, -0.5, -r3},
        {270, 0, -1},     {300, 0.5, -r3},  {315, r2, -r2},    {330, r3, -0.5}};
    bool hit = false;
    for (const Entry& e : table)
        if (e.deg == deg) { *c = (float)e.c; *s = (float)e.s; hit = true; }
    return hit;
}

void cos_sin(float deg, float* c, float* s) {
    if (tabulated(deg, c, s)) return;
    const float rad = (float)(deg * 3.14159265358979323846264338327950288 / 180.0);
    *c = (float)std::cos((double)rad);
    *s = (float)std::sin((double)rad);
}
}  // namespace

void euler_matrix_host(const float e[3], float m[9]) {
    float cf, sf, cp, sp, ct, st;
    cos_sin(e[0], &cf, &sf);  // phi
    cos_sin(e[1], &cp, &sp);  // psi
    cos_sin(e[2], &ct, &st);  // theta
    m[0] = cp * cf - ct * sp * sf;
    m[1] = sp * cf + ct * cp * sf;
    m[2] = st * sf;
    m[3] = -cp * sf - ct * sp * cf;
    m[4] = -sp * sf + ct * cp * cf;
    m[5] = st * cf;
    m[6] = st * sp;
    m[7] = -st * cp;
    m[8] = ct;
}

}  // namespace tg

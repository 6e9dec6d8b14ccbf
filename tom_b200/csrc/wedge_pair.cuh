// Index pair of the Hermitian part of a centred wedge weight on the FFT grid.
#pragma once
#include "common.cuh"

namespace tg {

// The two source voxels of (W'(k) + W'(-k)) / 2 with W' = ifftshift(W):
// ifftshift(v) and ifftshift(-v) (all boxes hold fewer than 2^31 voxels).
TG_D void wedge_pair(int v, int nx, int ny, int nz, int& s1, int& s2) {
    const int i = v % nx, t = v / nx, j = t % ny, k = t / ny;
    const int hx = nx / 2, hy = ny / 2, hz = nz / 2;
    const int a1 = i + hx < nx ? i + hx : i + hx - nx, b1 = j + hy < ny ? j + hy : j + hy - ny,
              c1 = k + hz < nz ? k + hz : k + hz - nz;
    const int mi = i ? nx - i : 0, mj = j ? ny - j : 0, mk = k ? nz - k : 0;
    const int a2 = mi + hx < nx ? mi + hx : mi + hx - nx, b2 = mj + hy < ny ? mj + hy : mj + hy - ny,
              c2 = mk + hz < nz ? mk + hz : mk + hz - nz;
    s1 = a1 + nx * (b1 + ny * c1);
    s2 = a2 + nx * (b2 + ny * c2);
}

}  // namespace tg

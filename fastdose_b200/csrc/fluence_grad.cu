// fluence_grad.cu -- the fluence-smoothness operator D_b of one beam (host).
//
// fluenceGradInit (IMRTOpt/src/IMRTOptimize_var.cpp:59-180) forms, per beam,
// Dx = kron(I, Dxy) F and Dy = kron(Dxy, I) F with Dxy the forward difference
// (-1 at i, +1 at i+1, rows 0..n-2; DxyInit, IMRTOpt/src/IMRTEigenLoad.cpp:307-327)
// and F the 0/1 filter onto the beam's active beamlets, then keeps the rows
// whose two ends are both active (row sum ~ 0 and |row| sum > 0) and stacks
// [Dx; Dy].  Both products reduce to "pairs of horizontally, then vertically,
// adjacent active pixels", which is what is enumerated here directly, in the
// reference's row order (x pairs row-major over the fluence map, then y pairs).
#include <vector>

#include "../../include/fd2_opt.h"
#include "fd2_internal.cuh"

extern "C" int fd2_fluence_grad(int fluence_dim, const uint8_t* active, int64_t* rows, int64_t* nnz,
                                int64_t* offsets, int64_t* columns, float* values) {
    FD2_REQUIRE(fluence_dim > 0 && active && rows && nnz && offsets && columns && values, FD2_ERR_INVALID_ARGUMENT,
                "fluence_grad: bad argument");
    const int n = fluence_dim;
    std::vector<int64_t> beamlet(static_cast<size_t>(n) * n, -1);  // active pixel -> beamlet column
    int64_t n_active = 0;
    for (int p = 0; p < n * n; p++)
        if (active[p]) beamlet[p] = n_active++;
    int64_t r = 0, z = 0;
    offsets[0] = 0;
    auto pair = [&](int p0, int p1) {
        if (beamlet[p0] < 0 || beamlet[p1] < 0) return;
        columns[z] = beamlet[p0];
        values[z++] = -1.0f;
        columns[z] = beamlet[p1];
        values[z++] = 1.0f;
        offsets[++r] = z;
    };
    for (int y = 0; y < n; y++)  // horizontal neighbours
        for (int x = 0; x + 1 < n; x++) pair(y * n + x, y * n + x + 1);
    for (int y = 0; y + 1 < n; y++)  // vertical neighbours
        for (int x = 0; x < n; x++) pair(y * n + x, (y + 1) * n + x);
    *rows = r;
    *nnz = z;
    return FD2_OK;
}

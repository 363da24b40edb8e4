// Pieces of the absorbing-boundary update shared by the forward step (step.cu) and its
// adjoint (adjoint.cu).
#pragma once
#include "common.cuh"

namespace pb
{

// Closed-form 4x4 solve by 2x2 sub-determinants (the method credited at fdtd.cu:36), kept
// operation for operation so the boundary values round like the reference's.
template <typename R>
__device__ inline void solve4(const R a[4][4], const R b[4], R out[4])
{
    R s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
    R s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    R s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3];
    R s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    R s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3];
    R s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    R c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3];
    R c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    R c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2];
    R c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    R c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2];
    R c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    R invdet = 1.0 / (s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0);
    R inv[4][4];
    inv[0][0] = (a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3) * invdet;
    inv[0][1] = (-a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3) * invdet;
    inv[0][2] = (a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3) * invdet;
    inv[0][3] = (-a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3) * invdet;
    inv[1][0] = (-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1) * invdet;
    inv[1][1] = (a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1) * invdet;
    inv[1][2] = (-a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1) * invdet;
    inv[1][3] = (a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1) * invdet;
    inv[2][0] = (a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0) * invdet;
    inv[2][1] = (-a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0) * invdet;
    inv[2][2] = (a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0) * invdet;
    inv[2][3] = (-a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0) * invdet;
    inv[3][0] = (-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0) * invdet;
    inv[3][1] = (a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0) * invdet;
    inv[3][2] = (-a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0) * invdet;
    inv[3][3] = (a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0) * invdet;
#pragma unroll
    for (int i = 0; i < 4; i++)
    {
        out[i] = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            out[i] += inv[i][j] * b[j];
    }
}

// number of cells in the boundary layer of [1, res-2]^3 (a coordinate equal to 1 or res-2)
__host__ __device__ inline long long boundary_cells(int res)
{
    const long long m = res - 2;
    return 2 * m * m + 2 * (m - 2) * m + 2 * (m - 2) * (m - 2);
}

// i-th cell of the boundary layer of [1, res-2]^3: the two x faces, then the two y faces
// without their x edges, then the two z faces without x and y edges
__device__ inline void boundary_cell(int i, int res, int &x, int &y, int &z)
{
    const int m = res - 2, lo = 1, hi = res - 2;
    int f = 2 * m * m;
    if (i < f)
    {
        x = i < m * m ? lo : hi;
        int r = i % (m * m);
        y = lo + r / m;
        z = lo + r % m;
        return;
    }
    i -= f;
    f = 2 * (m - 2) * m;
    if (i < f)
    {
        int half = (m - 2) * m;
        y = i < half ? lo : hi;
        int r = i % half;
        x = lo + 1 + r / m;
        z = lo + r % m;
        return;
    }
    i -= f;
    int half = (m - 2) * (m - 2);
    z = i < half ? lo : hi;
    int r = i % half;
    x = lo + 1 + r / (m - 2);
    y = lo + 1 + r % (m - 2);
}

}  // namespace pb

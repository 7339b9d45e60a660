// qgrid.cu -- the displacement bins of the full-q-grid S(q,t), in a fixed
// order of summation.
//
// S(q) for every q of the N x N grid is the 2-D DFT of the bins
//   G(dr, dc) = sum over pairs (i, j) with (r_i - r_j, c_i - c_j) = (dr, dc)
//               mod N of  alpha C_ij - m_i . z_j
// (the single-q phase of llg_sqt_baseline.c:265-268 applied to every q).  The
// GEMM epilogues leave, for every tile (mb, nb) of bm x bn sites, the sums of
// that value along each diagonal d = r - c of the tile (r, c the local row and
// column), split by class: 0 when c_j <= c_i (i - j needs no column wrap),
// 1 otherwise.  Along a diagonal, i - j = delta is constant, so the column
// displacement is dc = delta mod N for both classes, and the row displacement
// is (delta - dc) / N in class 0 and one more in class 1.
//
// Tiles with the same key k = mb - (bn / bm) nb have the same i - j on each
// diagonal: delta = k bm + d.  So the bins follow in two fixed-order passes:
//   keys: ds[k][d][cls] = sum over the tiles of key k (mb ascending)
//   bins: G(dr, dc) = sum over the (delta, cls) that land there (at most 4)
//         and over the keys whose tiles hold that delta (ascending)
// with no atomics: the bins repeat bit for bit.
#include <cuda_runtime.h>

#include "asd_internal.h"

namespace asd {
namespace {

__device__ __forceinline__ long floordiv(long a, long b) {  // b > 0
    long q = a / b;
    return (a % b != 0 && a < 0) ? q - 1 : q;
}

__global__ void qgrid_keys_kernel(const double *__restrict__ tdiag, int num_m, int num_n, int bm,
                                  int bn, double *__restrict__ ds) {
    const int R = bn / bm, nd = bm + bn - 1;
    const long nkeys = num_m + (long)R * (num_n - 1);
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nkeys * nd * 2) return;
    const long key = idx / (nd * 2);
    const int rem = (int)(idx - key * nd * 2);  // d index * 2 + class
    const long kp = key - (long)R * (num_n - 1);  // mb - R nb
    // tiles: mb = kp (mod R), 0 <= mb < num_m, 0 <= nb = (mb - kp) / R < num_n
    long mb = kp >= 0 ? kp : ((kp % R) + R) % R;
    const long mb_end = kp + (long)R * num_n;  // nb < num_n
    double s = 0.0;
    for (; mb < num_m && mb < mb_end; mb += R) {
        const long nb = (mb - kp) / R;
        s += tdiag[(mb * num_n + nb) * nd * 2 + rem];
    }
    ds[idx] = s;
}

__global__ void qgrid_bins_kernel(const double *__restrict__ ds, int num_m, int num_n, int bm,
                                  int bn, int N, double *__restrict__ G) {
    const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= (long)N * N) return;
    const int R = bn / bm, nd = bm + bn - 1;
    const long kmin = -(long)R * (num_n - 1), kmax = num_m - 1;
    const int dy = (int)(b / N), dx = (int)(b % N);
    double s = 0.0;
    for (int cls = 0; cls < 2; ++cls)
        for (int w = 0; w < 2; ++w) {
            const long ry = w == 0 ? dy : dy - N;  // row displacement r_i - r_j
            if (ry <= -N) continue;
            const long delta = (long)N * ry + dx - (cls ? N : 0);  // i - j
            long k0 = -floordiv(-(delta - (bm - 1)), bm);          // ceil
            long k1 = floordiv(delta + bn - 1, bm);
            if (k0 < kmin) k0 = kmin;
            if (k1 > kmax) k1 = kmax;
            for (long k = k0; k <= k1; ++k) {
                const long d = delta - k * bm;  // in [-(bn - 1), bm - 1]
                s += ds[((k - kmin) * nd + (d + bn - 1)) * 2 + cls];
            }
        }
    G[b] = s;
}

}  // namespace

long qgrid_keys(int num_m, int num_n, int bm, int bn) {
    return num_m + (long)(bn / bm) * (num_n - 1);
}

cudaError_t launch_qgrid_bins(const double *tdiag, int num_m, int num_n, int bm, int bn, int lat_n,
                              double *ds, double *G, cudaStream_t st) {
    if (bn % bm != 0) return cudaErrorInvalidValue;
    const long n1 = qgrid_keys(num_m, num_n, bm, bn) * (bm + bn - 1) * 2;
    qgrid_keys_kernel<<<(unsigned)((n1 + 255) / 256), 256, 0, st>>>(tdiag, num_m, num_n, bm, bn, ds);
    const long n2 = (long)lat_n * lat_n;
    qgrid_bins_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(ds, num_m, num_n, bm, bn, lat_n, G);
    return cudaGetLastError();
}

}  // namespace asd

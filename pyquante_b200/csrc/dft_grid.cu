// Numerical-integration kernels of the DFT path (the reference's MG2 grid,
// PyQuante/MG2.py:50-250, with Becke's partitioning of
// PyQuante/MolecularGrid.py:228-263, and the SVWN functional of
// PyQuante/DFunctionals.py:76-138,319-389,603-623):
//   * becke_weights_kernel: the cell weight of every grid point
//     w = w_atomic P_owner / sum_j P_j, P_j = prod_{k != j} s(mu'_jk),
//     mu_jk = (|r - R_j| - |r - R_k|)/|R_j - R_k|, mu' = mu + a_jk (1 - mu^2),
//     s = (1 - f3(mu'))/2 with f3 three applications of 1.5 x - 0.5 x^3;
//   * grid_amps_kernel: basis amplitudes B[g][i] = N_i x^l y^m z^n
//     sum_p c_p exp(-alpha_p r^2) (CGBF.amp, PyQuante/CGBF.py:116-120) --
//     the HBM-bound write of the grid path;
//   * grid_rowdot_kernel: rho_g = sum_i (B D)_gi B_gi (MG2.bdb);
//   * xc_svwn_kernel: Slater exchange (X-alpha 2/3, per spin) plus VWN
//     correlation per point, weighted: w f_xc, w v_a, w v_b.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/pyquante_b200.h"

namespace {

__global__ void becke_weights_kernel(int npts, const double *__restrict__ pts, const int *__restrict__ owner, int nat,
                                     const double *__restrict__ atoms, const double *__restrict__ adj,
                                     double *__restrict__ w)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += gridDim.x * blockDim.x) {
        const double px = pts[4 * g], py = pts[4 * g + 1], pz = pts[4 * g + 2];
        double sum = 0.0, own = 0.0;
        const int o = owner[g];
        for (int j = 0; j < nat; ++j) {
            const double xj = atoms[3 * j], yj = atoms[3 * j + 1], zj = atoms[3 * j + 2];
            const double rjp = sqrt((px - xj) * (px - xj) + (py - yj) * (py - yj) + (pz - zj) * (pz - zj));
            double P = 1.0;
            for (int k = 0; k < nat && P != 0.0; ++k) {
                if (k == j) continue;
                const double xk = atoms[3 * k], yk = atoms[3 * k + 1], zk = atoms[3 * k + 2];
                const double rkp = sqrt((px - xk) * (px - xk) + (py - yk) * (py - yk) + (pz - zk) * (pz - zk));
                const double rjk = sqrt((xj - xk) * (xj - xk) + (yj - yk) * (yj - yk) + (zj - zk) * (zj - zk));
                double mu = (rjp - rkp) / rjk;
                mu += adj[j * nat + k] * (1.0 - mu * mu);
#pragma unroll
                for (int it = 0; it < 3; ++it) mu = 1.5 * mu - 0.5 * mu * mu * mu;
                P *= 0.5 * (1.0 - mu);
            }
            sum += P;
            if (j == o) own = P;
        }
        w[g] = sum > 0.0 ? pts[4 * g + 3] * own / sum : 0.0;
    }
}

__global__ void grid_amps_kernel(int n, const double *__restrict__ origin, const int *__restrict__ powers,
                                 const int *__restrict__ prim_off, const double *__restrict__ exps,
                                 const double *__restrict__ cn, const double *__restrict__ norms, int npts,
                                 const double *__restrict__ pts, double *__restrict__ B)
{
    const int64_t total = (int64_t)npts * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(t / n), i = (int)(t - (int64_t)g * n);
        const double dx = pts[4 * g] - origin[3 * i], dy = pts[4 * g + 1] - origin[3 * i + 1],
                     dz = pts[4 * g + 2] - origin[3 * i + 2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        double poly = 1.0;
        for (int k = 0; k < powers[3 * i]; ++k) poly *= dx;
        for (int k = 0; k < powers[3 * i + 1]; ++k) poly *= dy;
        for (int k = 0; k < powers[3 * i + 2]; ++k) poly *= dz;
        double s = 0.0;
        for (int p = prim_off[i]; p < prim_off[i + 1]; ++p) s += cn[p] * exp(-exps[p] * r2);
        B[t] = norms[i] * poly * s;
    }
}

// one warp per row g: out[g] = sum_i A[g][i] B[g][i]
__global__ void grid_rowdot_kernel(int npts, int n, const double *__restrict__ A, const double *__restrict__ B,
                                   double *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < npts; g += (gridDim.x * blockDim.x) >> 5) {
        const double *a = A + (int64_t)g * n, *b = B + (int64_t)g * n;
        double s = 0.0;
        for (int i = lane; i < n; i += 32) s = fma(__ldg(a + i), __ldg(b + i), s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) out[g] = s;
    }
}

__device__ __forceinline__ double vwn_xx(double x, double b, double c) { return x * x + b * x + c; }

__device__ double vwn_eps(double x, double a, double x0, double b, double c)
{
    const double q = sqrt(4.0 * c - b * b);
    return a * (log(x * x / vwn_xx(x, b, c)) - b * (x0 / vwn_xx(x0, b, c)) * log((x - x0) * (x - x0) / vwn_xx(x, b, c)) +
                (2.0 * b / q) * (1.0 - (x0 * (2.0 * x0 + b) / vwn_xx(x0, b, c))) * atan(q / (2.0 * x + b)));
}

__device__ double vwn_deps(double x, double a, double x0, double b, double c)
{
    const double q = sqrt(4.0 * c - b * b), t = 2.0 * x + b;
    return a * (2.0 / x - t / vwn_xx(x, b, c) - 4.0 * b / (t * t + q * q) -
                (b * x0 / vwn_xx(x0, b, c)) * (2.0 / (x - x0) - t / vwn_xx(x, b, c) - 4.0 * (2.0 * x0 + b) / (t * t + q * q)));
}

// VWN parameters (A, x0, b, c) of the paramagnetic and ferromagnetic fits
// (Vosko, Wilk and Nusair, Can. J. Phys. 58, 1200 (1980)), as the reference uses them
#define VWN_P 0.0310907, -0.10498, 3.72744, 12.9352
#define VWN_F 0.01554535, -0.32500, 7.06042, 13.0045

__global__ void xc_svwn_kernel(int npts, const double *__restrict__ rhoa, const double *__restrict__ rhob,
                               const double *__restrict__ w, double *__restrict__ wf, double *__restrict__ wva,
                               double *__restrict__ wvb)
{
    const double tol = 1e-10;
    const double fac = -2.25 * (2.0 / 3.0) * cbrt(3.0 / (4.0 * M_PI));
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += gridDim.x * blockDim.x) {
        const double na = rhoa[g], nb = rhob[g];
        double f = 0.0, va = 0.0, vb = 0.0;
        // Slater exchange, per spin
        {
            const double ra = na < tol ? 0.0 : na, rb = nb < tol ? 0.0 : nb;
            const double a3 = cbrt(ra), b3 = cbrt(rb);
            f = fac * (ra * a3 + rb * b3);
            va = (4.0 / 3.0) * fac * a3;
            vb = (4.0 / 3.0) * fac * b3;
        }
        // VWN correlation
        const double rho = na + nb;
        if (rho >= tol) {
            const double zeta = (na - nb) / rho;
            const double x = pow(3.0 / (4.0 * M_PI) / rho, 1.0 / 6.0);
            const double ep = vwn_eps(x, VWN_P), dep = vwn_deps(x, VWN_P);
            const double gz = 1.125 * (pow(1.0 + zeta, 4.0 / 3.0) + pow(1.0 - zeta, 4.0 / 3.0) - 2.0);
            if (gz < tol) {
                f += ep * rho;
                va += ep - (x / 6.0) * dep;
                vb += ep - (x / 6.0) * dep;
            } else {
                const double ef = vwn_eps(x, VWN_F), def = vwn_deps(x, VWN_F);
                const double e = ep + gz * (ef - ep);
                const double dg = 1.5 * (cbrt(1.0 + zeta) - cbrt(1.0 - zeta));
                const double dx = dep + gz * (def - dep), dgg = (ef - ep) * dg;
                f += e * rho;
                va += e - (x / 6.0) * dx + dgg * (1.0 - zeta);
                vb += e - (x / 6.0) * dx - dgg * (1.0 + zeta);
            }
        }
        wf[g] = w[g] * f;
        wva[g] = w[g] * va;
        wvb[g] = w[g] * vb;
    }
}

int grid_of(int64_t total, int per)
{
    const int64_t g = (total + per - 1) / per;
    return (int)(g < 148 * 32 ? (g > 0 ? g : 1) : 148 * 32);
}

}  // namespace

extern "C" {

int pqb_becke_weights(int npts, const double *pts, const int *owner, int natoms, const double *atom_xyz,
                      const double *adjust, double *w, void *stream)
{
    if (npts < 0 || natoms <= 0 || !pts || !owner || !atom_xyz || !adjust || !w) return PQB_E_ARG;
    if (npts == 0) return PQB_OK;
    becke_weights_kernel<<<grid_of(npts, 128), 128, 0, (cudaStream_t)stream>>>(npts, pts, owner, natoms, atom_xyz,
                                                                             adjust, w);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_grid_amps(int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                  const double *cn, const double *norms, int npts, const double *pts, double *B, void *stream)
{
    if (n <= 0 || npts < 0 || !origin || !powers || !prim_off || !exps || !cn || !norms || !pts || !B)
        return PQB_E_ARG;
    if (npts == 0) return PQB_OK;
    grid_amps_kernel<<<grid_of((int64_t)npts * n, 256), 256, 0, (cudaStream_t)stream>>>(n, origin, powers, prim_off,
                                                                                         exps, cn, norms, npts, pts, B);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_grid_rowdot(int npts, int n, const double *A, const double *B, double *out, void *stream)
{
    if (npts < 0 || n <= 0 || !A || !B || !out) return PQB_E_ARG;
    if (npts == 0) return PQB_OK;
    grid_rowdot_kernel<<<grid_of((int64_t)npts * 32, 256), 256, 0, (cudaStream_t)stream>>>(npts, n, A, B, out);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_xc_svwn(int npts, const double *rhoa, const double *rhob, const double *w, double *wf, double *wva,
                double *wvb, void *stream)
{
    if (npts < 0 || !rhoa || !rhob || !w || !wf || !wva || !wvb) return PQB_E_ARG;
    if (npts == 0) return PQB_OK;
    xc_svwn_kernel<<<grid_of(npts, 128), 128, 0, (cudaStream_t)stream>>>(npts, rhoa, rhob, w, wf, wva, wvb);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

}  // extern "C"

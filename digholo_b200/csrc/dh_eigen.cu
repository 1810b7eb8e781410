// FP64 eigenvalues (and the eigenvectors of the smallest and largest) of a
// Hermitian matrix on the GPU, for the power meter: the squared singular
// values of the batch coefficient matrix that digHolo takes from cgesvd
// (svdSingularValues, digHolo.cpp:3021-3055; digHoloPowerMeter
// digHolo.cpp:11012-11062) are the eigenvalues of its FP64 Gram matrix, and
// MDL = s_min^2 / s_max^2 needs only their extremes -- and for its gradient
// the two extreme eigenvectors.
//
// One CTA (1024 threads) per matrix:
//   1. Householder tridiagonalisation, A = Q T Q^H, Q = H_0 H_1 ... H_{n-2},
//      H_k = I - tau_k v_k v_k^H with v_k[k+1] = 1 (the reflector convention
//      of LAPACK's zlarfg / zhetd2, lower triangle).  The matrix stays in
//      global memory (L2-resident for the sizes here, column-major); the
//      rank-2 update of step k - 1 is applied in the same pass that forms
//      A v_k for step k, so each step reads and writes the trailing block
//      once.
//   2. All eigenvalues of the real symmetric tridiagonal T (the reflectors
//      make every off-diagonal real) by Sturm-count bisection, one
//      eigenvalue per thread, ascending.
//   3. On request, inverse iteration on T for the smallest and largest
//      eigenvalue (tridiagonal LU with partial pivoting, one thread each),
//      then u = Q z by applying the reflectors in reverse order (one warp
//      each).
// Nothing waits on another CTA or on memory flags: no spin-waits.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>

namespace {

constexpr int NT = 1024;

__device__ __forceinline__ double2 cmulD(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ double2 cmulcD(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Sum over the block; every thread gets the result.  red holds 33 entries.
__device__ double2 blockSum(double2 v, double2* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double2 w = lane < (int)(blockDim.x >> 5) ? red[lane] : make_double2(0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
            w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
        }
        if (lane == 0) red[32] = w;
    }
    __syncthreads();
    const double2 r = red[32];
    __syncthreads();
    return r;
}

__device__ double blockMinMax(double v, double* red, bool isMax) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = isMax ? fmax(v, u) : fmin(v, u);
    }
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = lane < (int)(blockDim.x >> 5) ? red[lane] : (isMax ? -DBL_MAX : DBL_MAX);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(0xffffffffu, w, o);
            w = isMax ? fmax(w, u) : fmin(w, u);
        }
        if (lane == 0) red[32] = w;
    }
    __syncthreads();
    const double r = red[32];
    __syncthreads();
    return r;
}

// Number of eigenvalues of the tridiagonal (D, E2 = off-diagonal squared)
// below x (Sturm sequence with the pivot safeguard of LAPACK's dstebz).
__device__ int sturmCount(const double* D, const double* E2, int n, double x, double pivmin) {
    int cnt = 0;
    double q = D[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) cnt++;
    for (int i = 1; i < n; i++) {
        q = (D[i] - x) - E2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0) cnt++;
    }
    return cnt;
}

struct HeevArgs {
    double2* G;         // [count][n][n] column-major (element (i, j) at j n + i); overwritten
    int n;
    double* W;          // [count][n] eigenvalues, ascending
    double2* vecs;      // [count][2][n]: eigenvectors of the smallest and largest eigenvalue, or null
    double2* tau;       // [count][n] work
    double* lu;         // [count][2][6 n] work (inverse iteration)
    int extremes;       // 1: only W[0] and W[n-1] (the other entries untouched)
    double* trace;      // [count] sum of the eigenvalues (the tridiagonal's diagonal sum), or null
};

__global__ void __launch_bounds__(NT, 1) k_heev(HeevArgs a) {
    extern __shared__ double2 smem[];
    const int n = a.n, t = threadIdx.x;
    double2* A = a.G + (size_t)blockIdx.x * n * n;
    double2* tau = a.tau + (size_t)blockIdx.x * n;
    double2* vk = smem;             // reflector of this step, by row index
    double2* vp = vk + n;           // reflector of the previous step
    double2* xp = vp + n;           // w of the previous step (A22 -= v w^H + w v^H)
    double2* y = xp + n;            // A22 v
    double2* part = y + n;          // NT partial sums
    double* D = reinterpret_cast<double*>(part + NT);
    double* E = D + n;
    double* E2 = E + n;
    __shared__ double2 red[33];
    __shared__ double2 scal[2];
    __shared__ double redd[33];

    // ---- 1. tridiagonalisation
    bool havePrev = false;
    for (int k = 0; k + 1 < n; k++) {
        const int L = n - k - 1;
        double2* col = A + (size_t)k * n;
        // (a) the previous update on column k, rows k..n-1
        if (havePrev) {
            for (int i = k + t; i < n; i += NT) {
                const double2 u1 = cmulD(vp[i], make_double2(xp[k].x, -xp[k].y));
                const double2 u2 = cmulD(xp[i], make_double2(vp[k].x, -vp[k].y));
                double2 c = col[i];
                c.x -= u1.x + u2.x;
                c.y -= u1.y + u2.y;
                col[i] = c;
            }
        }
        __syncthreads();
        // (b) reflector for col[k+1 .. n-1]: alpha = col[k+1], x = col[k+2 ..]
        double2 s = make_double2(0.0, 0.0);
        for (int i = k + 2 + t; i < n; i += NT) s.x += col[i].x * col[i].x + col[i].y * col[i].y;
        s = blockSum(s, red);
        if (t == 0) {
            D[k] = col[k].x;
            const double2 alpha = col[k + 1];
            const double xnorm2 = s.x;
            double beta, tr, ti;
            double2 sc;
            if (xnorm2 == 0.0 && alpha.y == 0.0) {
                beta = alpha.x;
                tr = 0.0; ti = 0.0;
                sc = make_double2(0.0, 0.0);
            } else {
                const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
                beta = alpha.x >= 0.0 ? -nrm : nrm;
                tr = (beta - alpha.x) / beta;
                ti = -alpha.y / beta;
                // 1 / (alpha - beta)
                const double dr = alpha.x - beta, di = alpha.y;
                const double den = dr * dr + di * di;
                sc = make_double2(dr / den, -di / den);
            }
            E[k] = beta;
            E2[k] = beta * beta;
            tau[k] = make_double2(tr, ti);
            scal[0] = make_double2(tr, ti);
            scal[1] = sc;
        }
        __syncthreads();
        const double2 tk = scal[0], sc = scal[1];
        for (int i = k + 1 + t; i < n; i += NT) {
            double2 v;
            if (i == k + 1) {
                v = make_double2(1.0, 0.0);
            } else {
                v = cmulD(col[i], sc);
                col[i] = v;   // kept for the back-transformation
            }
            vk[i] = v;
        }
        __syncthreads();
        // (c) the previous update on the trailing block (rows, columns >= k+1)
        // fused with y = A22 v_k
        const int Lr = min(((L + 31) / 32) * 32, NT);
        const int groups = NT / Lr;
        for (int r0 = 0; r0 < L; r0 += Lr) {
            const int ri = r0 + (t % Lr), g = t / Lr;
            double2 acc = make_double2(0.0, 0.0);
            if (ri < L && g < groups) {
                const int i = k + 1 + ri;
                const double2 vpi = havePrev ? vp[i] : make_double2(0.0, 0.0);
                const double2 xpi = havePrev ? xp[i] : make_double2(0.0, 0.0);
                // CB columns per pass, their loads issued before any store:
                // the trailing block lives in L2, and one load in flight per
                // thread would leave each pass waiting on L2 latency CB times
                constexpr int CB = 4;
                for (int j0 = k + 1 + g; j0 < n; j0 += CB * groups) {
                    double2 e[CB];
#pragma unroll
                    for (int q = 0; q < CB; q++) {
                        const int j = j0 + q * groups;
                        e[q] = j < n ? A[(size_t)j * n + i] : make_double2(0.0, 0.0);
                    }
#pragma unroll
                    for (int q = 0; q < CB; q++) {
                        const int j = j0 + q * groups;
                        if (j >= n) break;
                        if (havePrev) {
                            const double2 u1 = cmulD(vpi, make_double2(xp[j].x, -xp[j].y));
                            const double2 u2 = cmulD(xpi, make_double2(vp[j].x, -vp[j].y));
                            e[q].x -= u1.x + u2.x;
                            e[q].y -= u1.y + u2.y;
                            A[(size_t)j * n + i] = e[q];
                        }
                        const double2 p = cmulD(e[q], vk[j]);
                        acc.x += p.x;
                        acc.y += p.y;
                    }
                }
            }
            part[t] = acc;
            __syncthreads();
            if (t < Lr && r0 + t < L) {
                double2 sum = make_double2(0.0, 0.0);
                for (int gg = 0; gg < groups; gg++) {
                    sum.x += part[gg * Lr + t].x;
                    sum.y += part[gg * Lr + t].y;
                }
                y[k + 1 + r0 + t] = sum;
            }
            __syncthreads();
        }
        // (d) x = tau y, alpha = -tau (x^H v) / 2, w = x + alpha v
        double2 d = make_double2(0.0, 0.0);
        for (int i = k + 1 + t; i < n; i += NT) {
            const double2 x = cmulD(tk, y[i]);
            y[i] = x;
            const double2 p = cmulcD(x, vk[i]);
            d.x += p.x;
            d.y += p.y;
        }
        d = blockSum(d, red);
        const double2 al = cmulD(make_double2(-0.5 * tk.x, -0.5 * tk.y), d);
        for (int i = k + 1 + t; i < n; i += NT) {
            const double2 w = cmulD(al, vk[i]);
            xp[i] = make_double2(y[i].x + w.x, y[i].y + w.y);
            vp[i] = vk[i];
        }
        havePrev = true;
        __syncthreads();
    }
    if (t == 0) {
        const int k = n - 1;
        double2 c = A[(size_t)k * n + k];
        if (havePrev) {
            const double2 u1 = cmulD(vp[k], make_double2(xp[k].x, -xp[k].y));
            const double2 u2 = cmulD(xp[k], make_double2(vp[k].x, -vp[k].y));
            c.x -= u1.x + u2.x;
        }
        D[k] = c.x;
        E[k] = 0.0;
        E2[k] = 0.0;
    }
    __syncthreads();

    // ---- 2. eigenvalues by bisection (Gershgorin interval)
    double lo = DBL_MAX, hi = -DBL_MAX, e2max = 0.0;
    for (int i = t; i < n; i += NT) {
        const double r = (i > 0 ? fabs(E[i - 1]) : 0.0) + (i + 1 < n ? fabs(E[i]) : 0.0);
        lo = fmin(lo, D[i] - r);
        hi = fmax(hi, D[i] + r);
        if (i + 1 < n) e2max = fmax(e2max, E2[i]);
    }
    lo = blockMinMax(lo, redd, false);
    hi = blockMinMax(hi, redd, true);
    e2max = blockMinMax(e2max, redd, true);
    const double scale = fmax(fabs(lo), fabs(hi));
    const double pivmin = DBL_MIN * fmax(1.0, e2max);
    const double tol = 4.0 * DBL_EPSILON * scale + 2.0 * pivmin;
    lo -= tol;
    hi += tol;
    double* W = a.W + (size_t)blockIdx.x * n;
    if (a.trace && t == 0) {
        double tr = 0.0;
        for (int i = 0; i < n; i++) tr += D[i];
        a.trace[blockIdx.x] = tr;
    }
    if (a.extremes) {
        // the smallest and the largest eigenvalue only (what MDL and its
        // gradient use): one warp each, 31 count points per pass, five bits
        // of the interval per Sturm count; every lane holds the same interval
        const int warp = t >> 5, lane = t & 31;
        if (warp < 2) {
            const int m = warp == 0 ? 0 : n - 1;
            double l = lo, h = hi;
            for (int it = 0; it < 100 && h - l > tol; it++) {
                const double step = (h - l) * (1.0 / 32.0);
                const double x = l + step * (double)(lane + 1);
                const bool above = lane < 31 && sturmCount(D, E2, n, x, pivmin) > m;
                const unsigned bits = __ballot_sync(0xffffffffu, above) & 0x7fffffffu;
                const int f = bits ? __ffs(bits) - 1 : 31;   // first count point above eigenvalue m
                const double nh = f < 31 ? l + step * (double)(f + 1) : h;
                const double nl = f > 0 ? l + step * (double)f : l;
                l = nl;
                h = nh;
            }
            if (lane == 0) W[m] = 0.5 * (l + h);
        }
    } else {
        // quadrisection, four lanes per eigenvalue: lanes 0-2 of a group
        // count at the interval's quarter points, the group keeps the
        // quarter holding eigenvalue m (two bits per Sturm count instead of
        // one).  Every lane of a group holds the same interval, so the
        // group's trip count is uniform.
        const int lane = t & 31, q4 = t & 3;
        const unsigned gmask = 0xFu << (lane & ~3);
        for (int m = t >> 2; m < n; m += NT / 4) {
            double l = lo, h = hi;
            for (int it = 0; it < 200 && h - l > tol; it++) {
                const double step = 0.25 * (h - l);
                const double x = l + step * (double)(q4 + 1);
                const bool above = q4 < 3 && sturmCount(D, E2, n, x, pivmin) > m;
                const unsigned bits = (__ballot_sync(gmask, above) >> (lane & ~3)) & 7u;
                const int f = bits ? __ffs(bits) - 1 : 3;   // first quarter point above eigenvalue m
                const double nh = f < 3 ? l + step * (double)(f + 1) : h;
                const double nl = f > 0 ? l + step * (double)f : l;
                l = nl;
                h = nh;
            }
            if (q4 == 0) W[m] = 0.5 * (l + h);
        }
    }
    if (!a.vecs) return;
    __syncthreads();

    // ---- 3. eigenvectors of the smallest and largest eigenvalue
    const int warp = t >> 5, lane = t & 31;
    if (warp >= 2) return;
    const double sigma = W[warp == 0 ? 0 : n - 1];
    double2* u = a.vecs + ((size_t)blockIdx.x * 2 + warp) * n;
    double* lu = a.lu + ((size_t)blockIdx.x * 2 + warp) * 6 * n;
    double* dl = lu;
    double* dd = lu + n;
    double* du = lu + 2 * n;
    double* du2 = lu + 3 * n;
    double* z = lu + 4 * n;
    int* piv = reinterpret_cast<int*>(lu + 5 * n);
    if (lane == 0) {
        const double tiny = DBL_EPSILON * fmax(scale, DBL_MIN);
        for (int i = 0; i < n; i++) {
            dd[i] = D[i] - sigma;
            if (i + 1 < n) { dl[i] = E[i]; du[i] = E[i]; }
            du2[i] = 0.0;
        }
        // LU with partial pivoting (the elimination of LAPACK's dgttrf)
        for (int i = 0; i + 1 < n; i++) {
            if (fabs(dd[i]) >= fabs(dl[i])) {
                piv[i] = i;
                if (dd[i] == 0.0) dd[i] = tiny;
                const double f = dl[i] / dd[i];
                dl[i] = f;
                dd[i + 1] -= f * du[i];
            } else {
                piv[i] = i + 1;
                const double f = dd[i] / dl[i];
                dd[i] = dl[i];
                dl[i] = f;
                const double tmp = du[i];
                du[i] = dd[i + 1];
                dd[i + 1] = tmp - f * dd[i + 1];
                if (i + 2 < n) {
                    du2[i] = du[i + 1];
                    du[i + 1] = -f * du[i + 1];
                }
            }
        }
        if (dd[n - 1] == 0.0) dd[n - 1] = tiny;
        for (int i = 0; i < n; i++) z[i] = 1.0 + 0.5 * (double)((i * 7919) % 97) / 97.0;
        for (int rep = 0; rep < 3; rep++) {
            for (int i = 0; i + 1 < n; i++) {
                if (piv[i] == i) {
                    z[i + 1] -= dl[i] * z[i];
                } else {
                    const double tmp = z[i];
                    z[i] = z[i + 1];
                    z[i + 1] = tmp - dl[i] * z[i];
                }
            }
            z[n - 1] /= dd[n - 1];
            if (n > 1) z[n - 2] = (z[n - 2] - du[n - 2] * z[n - 1]) / dd[n - 2];
            for (int i = n - 3; i >= 0; i--) z[i] = (z[i] - du[i] * z[i + 1] - du2[i] * z[i + 2]) / dd[i];
            double nrm = 0.0;
            for (int i = 0; i < n; i++) nrm = fmax(nrm, fabs(z[i]));
            if (!(nrm > 0.0) || !isfinite(nrm)) {
                for (int i = 0; i < n; i++) z[i] = (i == (warp == 0 ? 0 : n - 1)) ? 1.0 : 0.0;
                break;
            }
            for (int i = 0; i < n; i++) z[i] /= nrm;
        }
    }
    __syncwarp();
    // u = H_0 H_1 ... H_{n-2} z, normalised
    for (int i = lane; i < n; i += 32) u[i] = make_double2(z[i], 0.0);
    __syncwarp();
    for (int k = n - 2; k >= 0; k--) {
        const double2* col = A + (size_t)k * n;
        double2 d = make_double2(0.0, 0.0);
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double2 v = i == k + 1 ? make_double2(1.0, 0.0) : col[i];
            const double2 p = cmulcD(v, u[i]);
            d.x += p.x;
            d.y += p.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d.x += __shfl_xor_sync(0xffffffffu, d.x, o);
            d.y += __shfl_xor_sync(0xffffffffu, d.y, o);
        }
        const double2 td = cmulD(tau[k], d);
        __syncwarp();
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double2 v = i == k + 1 ? make_double2(1.0, 0.0) : col[i];
            const double2 p = cmulD(v, td);
            u[i].x -= p.x;
            u[i].y -= p.y;
        }
        __syncwarp();
    }
    double nn = 0.0;
    for (int i = lane; i < n; i += 32) nn += u[i].x * u[i].x + u[i].y * u[i].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
    const double inv = nn > 0.0 ? 1.0 / sqrt(nn) : 0.0;
    for (int i = lane; i < n; i += 32) u[i] = make_double2(u[i].x * inv, u[i].y * inv);
}

size_t heevSmem(int n) { return sizeof(double2) * (4 * (size_t)n + NT) + sizeof(double) * 3 * (size_t)n; }

}  // namespace

// Work buffers of the eigen solver, grown on demand and owned by the caller.
struct DhEigen {
    void* work = nullptr;
    size_t bytes = 0;
};

static int ensureWork(DhEigen& e, size_t need) {
    if (need <= e.bytes && e.work) return 0;
    if (e.work) cudaFree(e.work);
    e.work = nullptr;
    e.bytes = 0;
    if (cudaMalloc(&e.work, need) != cudaSuccess) return 1;
    e.bytes = need;
    return 0;
}

// Largest matrix the one-CTA solver takes (its shared memory).
int dh_eigen_max_n() { return 2048; }

// `count` Hermitian n x n matrices G (column-major, consecutive, overwritten):
// eigenvalues ascending into W[count][n]; with vecs non-null the unit
// eigenvectors of the smallest and the largest eigenvalue into
// vecs[count][2][n] (complex double).
int dh_eigen_solve(DhEigen& e, void* G, int n, int count, double* W, void* vecs, cudaStream_t s, int extremes = 0,
                   double* trace = nullptr) {
    if (n < 1 || n > dh_eigen_max_n() || count < 1) return 2;
    const size_t need = (size_t)count * n * sizeof(double2) + (size_t)count * 2 * 6 * n * sizeof(double);
    if (ensureWork(e, need)) return 3;
    HeevArgs a;
    a.G = static_cast<double2*>(G);
    a.n = n;
    a.W = W;
    a.vecs = static_cast<double2*>(vecs);
    a.tau = static_cast<double2*>(e.work);
    a.lu = reinterpret_cast<double*>(static_cast<char*>(e.work) + (size_t)count * n * sizeof(double2));
    a.extremes = extremes;
    a.trace = trace;
    const size_t smem = heevSmem(n);
    static size_t smemSet = 0;
    if (smem > 48 * 1024 && smem > smemSet) {
        if (cudaFuncSetAttribute(k_heev, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 4;
        smemSet = smem;
    }
    k_heev<<<count, NT, smem, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : 5;
}

int dh_eigen_values(DhEigen& e, void* G, int n, double* W, cudaStream_t s) {
    return dh_eigen_solve(e, G, n, 1, W, nullptr, s);
}

// The smallest and largest eigenvalue (W[0], W[n-1]; the other entries of W
// untouched), with vecs non-null their eigenvectors, and the eigenvalue sum.
int dh_eigen_extremes(DhEigen& e, void* G, int n, int count, double* W, void* vecs, double* trace, cudaStream_t s) {
    return dh_eigen_solve(e, G, n, count, W, vecs, s, 1, trace);
}

DhEigen* dh_eigen_create() { return new DhEigen(); }
void dh_eigen_destroy(DhEigen* e) {
    if (e) {
        if (e->work) cudaFree(e->work);
        delete e;
    }
}

extern "C" {

// Eigenvalues of one Hermitian n x n matrix given in host memory
// (column-major complex double, interleaved re/im), ascending into W (host);
// with vecs non-null the unit eigenvectors of the smallest and largest
// eigenvalue into vecs[2][n] complex (host).  A utility around the power
// meter's solver; runs on the current device and waits for it.
// No counterpart in the reference (its power meter calls LAPACK cgesvd).
int digHoloB200EigenHermitian(int n, const double* G, double* W, double* vecs) {
    if (n < 1 || n > dh_eigen_max_n()) return 5;   // DIGHOLO_ERROR_INVALIDDIMENSION
    if (!G || !W) return 3;                         // DIGHOLO_ERROR_NULLPOINTER
    DhEigen e;
    void* dG = nullptr;
    double* dW = nullptr;
    void* dV = nullptr;
    const size_t gb = (size_t)n * n * sizeof(double2);
    int rc = 0;
    if (cudaMalloc(&dG, gb) != cudaSuccess || cudaMalloc(&dW, n * sizeof(double)) != cudaSuccess ||
        (vecs && cudaMalloc(&dV, 2 * (size_t)n * sizeof(double2)) != cudaSuccess)) {
        rc = 9;                                     // DIGHOLO_ERROR_MEMORYALLOCATION
    } else if (cudaMemcpy(dG, G, gb, cudaMemcpyHostToDevice) != cudaSuccess ||
               dh_eigen_solve(e, dG, n, 1, dW, dV, 0) != 0 || cudaDeviceSynchronize() != cudaSuccess ||
               cudaMemcpy(W, dW, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
               (vecs && cudaMemcpy(vecs, dV, 2 * (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost) != cudaSuccess)) {
        rc = 1;
    }
    if (dG) cudaFree(dG);
    if (dW) cudaFree(dW);
    if (dV) cudaFree(dV);
    if (e.work) cudaFree(e.work);
    return rc;
}

}  // extern "C"

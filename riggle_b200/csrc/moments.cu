// Sliding-window moments of a source's coverage on one chromosome (K4-K7): build_depth_signal
// (src/fourier/depth.rs:109-215) and moments_from_signal (src/fourier/moments.rs:192-466).
//
// K4  depth signal g[0..N) in f32, bit for bit the reference's: the fractional-bin impulses are
//     summed per bin in the reference's order (all start spikes, then all end spikes, each in input
//     order) and the prefix sum follows simd_cumsum_f32's chunk-of-8 order, including its
//     sequential f32 carry chain (only chunks with a non-zero total change the carry, so the chain
//     runs over the compacted non-zero totals).  The f32 rounding residues of g move large-window
//     means by ~1e-4 relative, so any other summation order could not match the reference.
// K5  centred signal u = g - mean(g) in f64 and its prefix sum U (double-double scan).
// K6  autocorrelation A[m] = sum_k u[k] u[k+m] by a hand-written Stockham FFT (radix 16/8/4/2
//     passes, FP64): FFT(u zero-padded to 2^ceil(log2 2N)), |X|^2, FFT again, real part / M.
// K7  window moments for the L grid of the compact store:
//       sum_j F_L(j)   = (UU(N+1) - UU(L)) - UU(N-L+1)                    (UU = prefix of U)
//       sum_j F_L(j)^2 = L A[0] + 2 (L P0(L) - P1(L)) - Q(L-1) - V(L-1)
//     with F_L(j) the window sums of u, P0/P1 prefix sums of A[m] and m A[m] (m >= 1), Q the prefix
//     sum of U[t]^2 and V that of (U[N] - U[N-t])^2 (the partial windows at both ends of the full
//     linear convolution).  mean(L) = L mean(g) + sum F / n_w, var(L) = sum F^2 / n_w - (sum F /
//     n_w)^2 in FP64, clamped at 0 as the reference does.  Every term is bounded by the centred
//     signal, so the cancellation that the reference's d*-autocorrelation suffers (~1e10,
//     docs/todo.md) does not arise; all prefix sums are double-double (compensated two-sum).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace rgl {

std::vector<uint64_t> moment_grid(uint64_t n);

struct DD {
    double hi, lo;
};
__host__ __device__ __forceinline__ DD dd_two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return DD{s, e};
}
__host__ __device__ __forceinline__ DD dd_add(DD a, DD b) {
    DD s = dd_two_sum(a.hi, b.hi);
    const DD t = dd_two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = dd_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return dd_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DD dd_neg(DD a) { return DD{-a.hi, -a.lo}; }
__device__ __forceinline__ DD dd_mul_d(DD a, double b) {
    const double p = a.hi * b;
    double e = fma(a.hi, b, -p);
    e = fma(a.lo, b, e);
    return dd_two_sum(p, e);
}
struct DDAdd {
    __device__ __forceinline__ DD operator()(const DD& a, const DD& b) const { return dd_add(a, b); }
};

// ---- K4: impulses ---------------------------------------------------------------------------------
__global__ void k_spike_records(uint32_t n, const rgl_interval* __restrict__ iv, uint32_t n_bins, uint32_t bin,
                                uint64_t* __restrict__ key, float* __restrict__ val) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t max_bp = n_bins * bin;  // build_spikes clip (src/fourier/depth.rs:206-215), u32 arithmetic
    for (uint32_t phase = 0; phase < 2; phase++) {
        const uint32_t x0 = phase ? iv[i].end : iv[i].start;
        const uint32_t x = x0 < max_bp ? x0 : max_bp;
        const uint32_t b = x / bin;
        const float frac = __fdiv_rn((float)(x % bin), (float)bin);
        const float c1 = __fsub_rn(1.0f, frac);
        const uint64_t base = ((uint64_t)phase << 32) | i;
        const uint64_t j = 4ull * i + 2 * phase;
        if (b < n_bins) {
            key[j] = ((uint64_t)b << 33) | base;
            val[j] = phase ? -c1 : c1;
        } else {
            key[j] = ~0ull;
            val[j] = 0.f;
        }
        if (frac > 0.0f && b + 1 < n_bins) {
            key[j + 1] = ((uint64_t)(b + 1) << 33) | base;
            val[j + 1] = phase ? -frac : frac;
        } else {
            key[j + 1] = ~0ull;
            val[j + 1] = 0.f;
        }
    }
}

// One thread per run of equal bins in the sorted records: the bin's impulse, summed in f32 in the
// reference's order.
__global__ void k_bin_sums(uint64_t m, const uint64_t* __restrict__ key, const float* __restrict__ val,
                           float* __restrict__ g) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= m || key[j] == ~0ull) return;
    const uint64_t b = key[j] >> 33;
    if (j > 0 && (key[j - 1] >> 33) == b) return;
    float s = 0.0f;
    for (uint64_t k = j; k < m && key[k] != ~0ull && (key[k] >> 33) == b; k++) s = __fadd_rn(s, val[k]);
    g[b] = s;
}

// ---- K4: simd_cumsum_f32 (src/fourier/depth.rs:143-204) in its own order ------------------------------
__global__ void k_chunk_local(uint64_t full, float* __restrict__ g, float* __restrict__ totals,
                              uint8_t* __restrict__ nz) {
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= full) return;
    float v[8];
    const float4* p = reinterpret_cast<const float4*>(g + 8 * c);
    const float4 a = p[0], b = p[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
#pragma unroll
    for (int i = 1; i < 8; i++) v[i] = __fadd_rn(v[i], v[i - 1]);
    float4* q = reinterpret_cast<float4*>(g + 8 * c);
    q[0] = make_float4(v[0], v[1], v[2], v[3]);
    q[1] = make_float4(v[4], v[5], v[6], v[7]);
    totals[c] = v[7];
    nz[c] = v[7] != 0.0f;
}

// The sequential f32 carry over the chunks whose total is non-zero (adding an exact zero leaves
// the carry unchanged), then the tail elements, exactly as the reference orders them.
__global__ void k_carry_chain(const int* __restrict__ count, const uint32_t* __restrict__ idx,
                              const float* __restrict__ totals, float* __restrict__ cum_after, float* __restrict__ g,
                              uint64_t n, uint64_t full) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float carry = 0.0f;
    const int cnt = *count;
    for (int k = 0; k < cnt; k++) {
        carry = __fadd_rn(carry, totals[idx[k]]);
        cum_after[k] = carry;
    }
    const uint64_t tail = full * 8;
    for (uint64_t i = tail + 1; i < n; i++) g[i] = __fadd_rn(g[i], g[i - 1]);
    if (full > 0 && tail < n && carry != 0.0f)
        for (uint64_t i = tail; i < n; i++) g[i] = __fadd_rn(g[i], carry);
}

__global__ void k_apply_carry(uint64_t full, const int* __restrict__ count, const uint32_t* __restrict__ idx,
                              const float* __restrict__ cum_after, float* __restrict__ g) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= full * 8) return;
    const uint64_t c = i >> 3;
    if (c == 0) return;  // the reference adds no carry to chunk 0
    // carries[c] = running sum of the totals of chunks < c = cum_after of the last non-zero chunk < c
    int lo = 0, hi = *count;  // number of compacted chunks with index < c
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (idx[mid] < c) lo = mid + 1; else hi = mid;
    }
    const float carry = lo ? cum_after[lo - 1] : 0.0f;
    g[i] = __fadd_rn(g[i], carry);
}

// ---- K5 ---------------------------------------------------------------------------------------------
__global__ void k_to_dd(uint64_t n, const float* __restrict__ g, DD* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = DD{(double)g[i], 0.0};
}

// u = g - gbar into the zero-padded complex FFT input and a DD array (u[N] = 0) for the U scan.
__global__ void k_center(uint64_t n, uint64_t M, const float* __restrict__ g, const DD* __restrict__ gsum,
                         double2* __restrict__ x, DD* __restrict__ udd) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= M) return;
    const double gbar = gsum->hi / (double)n + gsum->lo / (double)n;
    const double u = i < n ? (double)g[i] - gbar : 0.0;
    x[i] = make_double2(u, 0.0);
    if (i <= n) udd[i] = DD{i < n ? u : 0.0, 0.0};
}

__global__ void k_dd_to_double(uint64_t n, const DD* __restrict__ in, double* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i].hi + in[i].lo;
}

// ---- K6: Stockham FFT (FP64) ----------------------------------------------------------------------
// One pass of the out-of-place Stockham formulation (Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC 2008): thread j loads R elements at stride M/R,
// twiddles them by exp(-2 pi i (j mod Ns) r / (Ns R)), applies a radix-R DFT in registers and
// stores them at (j / Ns) Ns R + (j mod Ns) + r Ns.  log_R passes with Ns = 1, R, R^2, ... leave the
// transform in natural order.
__constant__ double2 c_tw16[16];  // exp(-2 pi i k / 16), k < 16 (host-computed)

template <int R>
__device__ __forceinline__ void dft_regs(double2* v) {
    // in-register radix-2 DIT on R = 2^r points (bit-reversed input order, natural output)
#pragma unroll
    for (int i = 0; i < R; i++) {
        int j = 0;
#pragma unroll
        for (int b = 1; b < R; b <<= 1) j = (j << 1) | ((i / b) & 1);
        if (i < j) {
            const double2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += len) {
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                const double2 w = c_tw16[k * (16 / len)];
                const double2 a = v[i + k], b = v[i + k + len / 2];
                const double2 t = make_double2(b.x * w.x - b.y * w.y, b.x * w.y + b.y * w.x);
                v[i + k] = make_double2(a.x + t.x, a.y + t.y);
                v[i + k + len / 2] = make_double2(a.x - t.x, a.y - t.y);
            }
        }
    }
}

template <int R>
__global__ void __launch_bounds__(256) k_fft_pass(const double2* __restrict__ in, double2* __restrict__ out,
                                                  uint64_t M, uint64_t Ns) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = M / R;
    if (j >= stride) return;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[j + r * stride];
    const uint64_t k = j % Ns;
    if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) {
            // angle -2 pi k r / (Ns R), as sincospi of the exact rational -2 k r / (Ns R)
            double s, c;
            sincospi(-2.0 * (double)(k * r) / (double)(Ns * R), &s, &c);
            const double2 a = v[r];
            v[r] = make_double2(a.x * c - a.y * s, a.x * s + a.y * c);
        }
    }
    dft_regs<R>(v);
    const uint64_t base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[base + r * Ns] = v[r];
}

__global__ void k_power(uint64_t M, double2* __restrict__ x) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < M) {
        const double2 a = x[i];
        x[i] = make_double2(a.x * a.x + a.y * a.y, 0.0);
    }
}

// ---- K7 -----------------------------------------------------------------------------------------
enum Term : int { T_A = 0, T_MA = 1, T_U2 = 2, T_V2 = 3, T_U = 4 };

// Scan inputs for the prefix sums: element t of term T (t = 0..len-1).
__global__ void k_term(uint64_t len, int term, const double2* __restrict__ y, double inv_m,
                       const double* __restrict__ U, uint64_t n, DD* __restrict__ out) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= len) return;
    double v = 0.0;
    switch (term) {
        case T_A: v = (t >= 1 && t < n) ? y[t].x * inv_m : 0.0; break;                  // A[t], t >= 1
        case T_MA: v = (t >= 1 && t < n) ? (double)t * (y[t].x * inv_m) : 0.0; break;  // t A[t]
        case T_U2: v = (t >= 1 && t <= n) ? U[t] * U[t] : 0.0; break;                    // U[t]^2, t >= 1
        case T_V2: {                                                                   // (U[N]-U[N-t])^2
            if (t >= 1 && t < n) {
                const double d = U[n] - U[n - t];
                v = d * d;
            }
            break;
        }
        default: v = (t <= n) ? U[t] : 0.0;  // U[t]
    }
    out[t] = DD{v, 0.0};
}

// Gathers inclusive prefix values at the requested indices (pre[i] = sum of terms 0..i).
__global__ void k_gather(uint32_t k, const uint64_t* __restrict__ at, const DD* __restrict__ pre, DD* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) out[i] = pre[at[i]];
}

// Windows with few positions (nw = N - L + 1 small, L close to N): the window sums F_L(j) then differ
// from one another by a small part of their size, and any formula that forms the second moment and
// subtracts the squared mean cancels (the reference's own f64 formula loses all digits there).
// These L are reduced directly: d_j = F_L(j) - F_L(0) = (U[j+L] - U[j]) - U[L] from the prefix sums
// U of the centred signal (U[0] = 0), summed with d_j^2 in double-double over the nw windows, and
// var = sum d^2 / nw - (sum d / nw)^2.  One block per such L; out[i] = var.
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e = fma(a.hi, b.lo, e);
    e = fma(a.lo, b.hi, e);
    return dd_two_sum(p, e);
}
__device__ __forceinline__ DD dd_div_d(DD a, double b) {
    const double q = a.hi / b;
    const DD r = dd_add(a, dd_neg(dd_mul_d(DD{q, 0.0}, b)));
    return dd_two_sum(q, (r.hi + r.lo) / b);
}
template <typename UT>
__device__ __forceinline__ DD u_at(const UT* U, uint64_t i);
template <>
__device__ __forceinline__ DD u_at<double>(const double* U, uint64_t i) { return DD{U[i], 0.0}; }
template <typename UT>
__global__ void __launch_bounds__(256) k_direct_var(const uint32_t* __restrict__ which, const uint64_t* __restrict__ ls,
                                                    uint64_t n, const UT* __restrict__ U, double uscale,
                                                    double* __restrict__ out) {
    const uint32_t i = which[blockIdx.x];
    const uint64_t L = ls[i], nw = n - L + 1;
    const DD uL = u_at<UT>(U, L);
    DD s1{0.0, 0.0}, s2{0.0, 0.0};
    for (uint64_t j = threadIdx.x; j < nw; j += blockDim.x) {
        const DD d = dd_add(dd_add(u_at<UT>(U, j + L), dd_neg(u_at<UT>(U, j))), dd_neg(uL));
        s1 = dd_add(s1, d);
        s2 = dd_add(s2, dd_mul(d, d));
    }
    __shared__ DD r1[256], r2[256];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (uint32_t k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            r1[threadIdx.x] = dd_add(r1[threadIdx.x], r1[threadIdx.x + k]);
            r2[threadIdx.x] = dd_add(r2[threadIdx.x], r2[threadIdx.x + k]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const DD m1 = dd_div_d(r1[0], (double)nw), m2 = dd_div_d(r2[0], (double)nw);
        const DD v = dd_add(m2, dd_neg(dd_mul(m1, m1)));
        const double var = (v.hi + v.lo) * uscale * uscale;
        out[i] = var > 0.0 ? var : 0.0;
    }
}

__global__ void k_window_moments(uint32_t G, const uint64_t* __restrict__ ls, uint64_t n,
                                 const DD* __restrict__ gsum, double a0, const DD* __restrict__ P0,
                                 const DD* __restrict__ P1, const DD* __restrict__ Q, const DD* __restrict__ V,
                                 const DD* __restrict__ UU_L, const DD* __restrict__ UU_R, DD uu_total,
                                 float2* __restrict__ out, double* __restrict__ mean_out, double* __restrict__ var_out,
                                 const double* __restrict__ direct_var) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    const uint64_t L = ls[i];
    const double nw = (double)(n - L + 1);
    const double gbar = gsum->hi / (double)n + gsum->lo / (double)n;
    // sum_j F_L(j) = (UU(N+1) - UU(L)) - UU(N-L+1)
    const DD sf = dd_add(dd_add(uu_total, dd_neg(UU_L[i])), dd_neg(UU_R[i]));
    const double fbar = (sf.hi + sf.lo) / nw;
    // sum_j F_L(j)^2 = L A[0] + 2 (L P0 - P1) - Q - V
    DD s2 = DD{(double)L * a0, fma((double)L, a0, -(double)L * a0)};
    const DD inner = dd_add(dd_mul_d(P0[i], (double)L), dd_neg(P1[i]));
    s2 = dd_add(s2, dd_mul_d(inner, 2.0));
    s2 = dd_add(s2, dd_neg(Q[i]));
    s2 = dd_add(s2, dd_neg(V[i]));
    const double mean = (double)L * gbar + fbar;
    double var = (s2.hi + s2.lo) / nw - fbar * fbar;
    if (!(var > 0.0)) var = 0.0;
    if (direct_var && direct_var[i] >= 0.0) var = direct_var[i];  // few windows: reduced directly
    out[i] = make_float2((float)mean, (float)var);
    if (mean_out) mean_out[i] = mean;
    if (var_out) var_out[i] = var;
}

// ---- the compensated-FP32 path (K5-K7 with float-float arithmetic) ------------------------------
// Every value is an unevaluated sum hi + lo of two floats (|lo| <= ulp(hi) / 2), about 48 bits of
// significand, kept by the error-free transformations two-sum (Knuth) and two-product (one FMA)
// as in Dekker's double-length arithmetic (T. J. Dekker, "A floating-point technique for extending
// the available precision", Numer. Math. 18, 1971; Y. Hida, X. S. Li, D. H. Bailey, "Algorithms for
// quad-double precision floating point arithmetic", ARITH 2001, for the add / mul sequences).  The
// centred signal is scaled by a power of two per chromosome so that it is O(1) (no denormal lo
// parts), the FFT, the power spectrum and the prefix sums run in float-float, and FP64 appears only
// when the per-L results are combined (k_window_moments: the final reduction and the variance
// subtraction).
struct FF {
    float hi, lo;
};
struct CFF {
    FF re, im;
};
__device__ __forceinline__ FF ff_two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return FF{s, e};
}
__device__ __forceinline__ FF ff_quick(float a, float b) {  // |a| >= |b|
    const float s = __fadd_rn(a, b);
    return FF{s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ FF ff_add(FF a, FF b) {
    FF s = ff_two_sum(a.hi, b.hi);
    const FF t = ff_two_sum(a.lo, b.lo);
    s.lo = __fadd_rn(s.lo, t.hi);
    s = ff_quick(s.hi, s.lo);
    s.lo = __fadd_rn(s.lo, t.lo);
    return ff_quick(s.hi, s.lo);
}
__device__ __forceinline__ FF ff_neg(FF a) { return FF{-a.hi, -a.lo}; }
__device__ __forceinline__ FF ff_sub(FF a, FF b) { return ff_add(a, ff_neg(b)); }
__device__ __forceinline__ FF ff_mul(FF a, FF b) {
    const float p = __fmul_rn(a.hi, b.hi);
    float e = __fmaf_rn(a.hi, b.hi, -p);
    e = __fmaf_rn(a.hi, b.lo, e);
    e = __fmaf_rn(a.lo, b.hi, e);
    return ff_quick(p, e);
}
__device__ __forceinline__ FF ff_from_double_exact(uint64_t t) {  // an integer below 2^48, exactly
    const float hi = (float)(t & ~0xFFFFFFull);                    // the top bits (exact in a float)
    return ff_two_sum(hi, (float)(t & 0xFFFFFFull));
}
__device__ __forceinline__ CFF cff_add(CFF a, CFF b) { return CFF{ff_add(a.re, b.re), ff_add(a.im, b.im)}; }
__device__ __forceinline__ CFF cff_sub(CFF a, CFF b) { return CFF{ff_sub(a.re, b.re), ff_sub(a.im, b.im)}; }
__device__ __forceinline__ CFF cff_mul(CFF a, CFF b) {
    return CFF{ff_sub(ff_mul(a.re, b.re), ff_mul(a.im, b.im)), ff_add(ff_mul(a.re, b.im), ff_mul(a.im, b.re))};
}
struct FFAdd {
    __device__ __forceinline__ FF operator()(const FF& a, const FF& b) const { return ff_add(a, b); }
};
template <>
__device__ __forceinline__ DD u_at<FF>(const FF* U, uint64_t i) {
    return dd_two_sum((double)U[i].hi, (double)U[i].lo);
}

__constant__ CFF c_tw16f[16];  // exp(-2 pi i k / 16) as float-float (host-computed)

template <int R>
__device__ __forceinline__ void dft_regs_ff(CFF* v) {
#pragma unroll
    for (int i = 0; i < R; i++) {
        int j = 0;
#pragma unroll
        for (int b = 1; b < R; b <<= 1) j = (j << 1) | ((i / b) & 1);
        if (i < j) {
            const CFF t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += len) {
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                const CFF a = v[i + k];
                const CFF t = k == 0 ? v[i + k + len / 2] : cff_mul(v[i + k + len / 2], c_tw16f[k * (16 / len)]);
                v[i + k] = cff_add(a, t);
                v[i + k + len / 2] = cff_sub(a, t);
            }
        }
    }
}

// One Stockham pass as k_fft_pass, in float-float.  The twiddle exp(-2 pi i t / M), t = k r M / (Ns R),
// is the product of two table entries: wc[t >> tb] (coarse) and wf[t & (2^tb - 1)] (fine).
template <int R>
__global__ void __launch_bounds__(128) k_ff_fft_pass(const CFF* __restrict__ in, CFF* __restrict__ out, uint64_t M,
                                                     uint64_t Ns, const CFF* __restrict__ wc,
                                                     const CFF* __restrict__ wf, int tb) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = M / R;
    if (j >= stride) return;
    CFF v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[j + r * stride];
    const uint64_t k = j % Ns;
    if (Ns > 1) {
        const uint64_t step = M / (Ns * R);  // t = k r step < M
        const uint64_t mask = (1ull << tb) - 1;
#pragma unroll
        for (int r = 1; r < R; r++) {
            const uint64_t t = k * (uint64_t)r * step;
            const CFF w = cff_mul(wc[t >> tb], wf[t & mask]);
            v[r] = cff_mul(v[r], w);
        }
    }
    dft_regs_ff<R>(v);
    const uint64_t base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[base + r * Ns] = v[r];
}

// u = (g - gbar) 2^-e into the zero-padded complex input (u[N] = 0 for the U scan).
__global__ void k_ff_center(uint64_t n, uint64_t M, const float* __restrict__ g, const FF* __restrict__ gsum,
                            float scale, CFF* __restrict__ x, FF* __restrict__ u_out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= M) return;
    FF u = FF{0.f, 0.f};
    if (i < n) {
        // gbar = gsum / n in float-float: one Newton step on the float quotient
        const FF S = *gsum;
        const float q = __fdiv_rn(S.hi, (float)n);
        const FF qn = ff_mul(FF{q, 0.f}, ff_from_double_exact(n));
        const FF r = ff_sub(S, qn);
        const FF gbar = ff_quick(q, __fdiv_rn(r.hi, (float)n));
        u = ff_sub(FF{g[i], 0.f}, gbar);
        u = FF{u.hi * scale, u.lo * scale};  // exact: scale is a power of two
    }
    x[i] = CFF{u, FF{0.f, 0.f}};
    if (i <= n) u_out[i] = u;
}

__global__ void k_ff_from_float(uint64_t n, const float* __restrict__ g, FF* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = FF{g[i], 0.f};
}

__global__ void k_ff_power(uint64_t M, CFF* __restrict__ x) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < M) {
        const CFF a = x[i];
        x[i] = CFF{ff_add(ff_mul(a.re, a.re), ff_mul(a.im, a.im)), FF{0.f, 0.f}};
    }
}

// Scan inputs of the compensated path, as k_term (A[t] = Re Y[t] / M, an exact power-of-two scale).
__global__ void k_ff_term(uint64_t len, int term, const CFF* __restrict__ y, float inv_m, const FF* __restrict__ U,
                          uint64_t n, FF* __restrict__ out) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= len) return;
    FF v = FF{0.f, 0.f};
    switch (term) {
        case T_A:
            if (t >= 1 && t < n) v = FF{y[t].re.hi * inv_m, y[t].re.lo * inv_m};
            break;
        case T_MA:
            if (t >= 1 && t < n) v = ff_mul(ff_from_double_exact(t), FF{y[t].re.hi * inv_m, y[t].re.lo * inv_m});
            break;
        case T_U2:
            if (t >= 1 && t <= n) v = ff_mul(U[t], U[t]);
            break;
        case T_V2:
            if (t >= 1 && t < n) {
                const FF d = ff_sub(U[n], U[n - t]);
                v = ff_mul(d, d);
            }
            break;
        default:
            if (t <= n) v = U[t];
    }
    out[t] = v;
}

// Inclusive prefix values at the requested indices, widened to double-double and scaled back by
// the exact power of two 2^sc (the FP64 final reduction starts here).
__global__ void k_ff_gather(uint32_t k, const uint64_t* __restrict__ at, const FF* __restrict__ pre, int sc,
                            DD* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) {
        const FF v = pre[at[i]];
        out[i] = DD{ldexp((double)v.hi, sc), ldexp((double)v.lo, sc)};
    }
}

// U[0] = 0, U[s] = inclusive scan of u at s - 1.
__global__ void k_ff_shift(uint64_t n, const FF* __restrict__ incl, FF* __restrict__ U) {
    const uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s <= n) U[s] = s ? incl[s - 1] : FF{0.f, 0.f};
}

}  // namespace rgl

using namespace rgl;

// Per-build device workspace (grown on demand) and the host twiddle table.
namespace {
struct MomentWs {
    DevBuf iv, key_a, key_b, val_a, val_b, g, totals, nz, idx, cum, cnt, fa, fb, U, dd_in, dd_out, at, gl, outs, tmp,
        gsum, grid, mv, dv;
};
std::mutex g_ws_mu;
MomentWs g_ws[16];  // one workspace per device ordinal
bool g_tw_ready[64] = {false};

int upload_twiddles(int device) {
    if (device >= 0 && device < 64 && g_tw_ready[device]) return RGL_OK;
    double2 tw[16];
    for (int k = 0; k < 16; k++) tw[k] = make_double2(std::cos(2.0 * M_PI * k / 16.0), -std::sin(2.0 * M_PI * k / 16.0));
    RGL_CUDA(cudaMemcpyToSymbol(c_tw16, tw, sizeof(tw)));
    if (device >= 0 && device < 64) g_tw_ready[device] = true;
    return RGL_OK;
}

inline unsigned blocks_for(uint64_t n) { return (unsigned)((n + 255) / 256); }

// Bit-exact reference depth signal of n intervals into ws.g (N floats).
int depth_signal_dev(MomentWs& w, const rgl_interval* h_iv, uint64_t n, uint64_t N, uint32_t bin, cudaStream_t st) {
    RGL_TRY(w.g.ensure(std::max<uint64_t>(N, 8) * 4 + 64));
    RGL_CUDA(cudaMemsetAsync(w.g.p, 0, N * 4 + 64, st));
    if (n) {
        if (n >= (1ull << 29)) return fail(RGL_ERR_INVALID_ARGUMENT, "too many intervals for one depth signal");
        const uint64_t m = 4 * n;
        RGL_TRY(w.iv.ensure(n * sizeof(rgl_interval)));
        RGL_TRY(w.key_a.ensure(m * 8));
        RGL_TRY(w.key_b.ensure(m * 8));
        RGL_TRY(w.val_a.ensure(m * 4));
        RGL_TRY(w.val_b.ensure(m * 4));
        RGL_CUDA(cudaMemcpyAsync(w.iv.p, h_iv, n * sizeof(rgl_interval), cudaMemcpyHostToDevice, st));
        k_spike_records<<<blocks_for(n), 256, 0, st>>>((uint32_t)n, w.iv.as<rgl_interval>(), (uint32_t)N, bin,
                                                        w.key_a.as<uint64_t>(), w.val_a.as<float>());
        int bits = 33;
        while (bits < 64 && (1ull << (bits - 33)) <= N) bits++;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, w.key_a.as<uint64_t>(), w.key_b.as<uint64_t>(), w.val_a.as<float>(),
                                        w.val_b.as<float>(), (int)m, 0, 64, st);
        RGL_TRY(w.tmp.ensure(tb + 256));
        tb = w.tmp.cap;
        // all 64 bits: invalid records (~0) sort last
        RGL_CUDA(cub::DeviceRadixSort::SortPairs(w.tmp.p, tb, w.key_a.as<uint64_t>(), w.key_b.as<uint64_t>(),
                                                 w.val_a.as<float>(), w.val_b.as<float>(), (int)m, 0, 64, st));
        k_bin_sums<<<blocks_for(m), 256, 0, st>>>(m, w.key_b.as<uint64_t>(), w.val_b.as<float>(), w.g.as<float>());
    }
    if (N <= 1) return RGL_OK;
    const uint64_t full = N / 8;
    RGL_TRY(w.totals.ensure(full * 4 + 16));
    RGL_TRY(w.nz.ensure(full + 16));
    RGL_TRY(w.idx.ensure(full * 4 + 16));
    RGL_TRY(w.cum.ensure(full * 4 + 16));
    RGL_TRY(w.cnt.ensure(16));
    if (full) k_chunk_local<<<blocks_for(full), 256, 0, st>>>(full, w.g.as<float>(), w.totals.as<float>(), w.nz.as<uint8_t>());
    RGL_CUDA(cudaMemsetAsync(w.cnt.p, 0, 16, st));
    if (full) {
        size_t tb = 0;
        cub::DeviceSelect::Flagged(nullptr, tb, thrust::counting_iterator<uint32_t>(0), w.nz.as<uint8_t>(),
                                   w.idx.as<uint32_t>(), w.cnt.as<int>(), (int)full, st);
        RGL_TRY(w.tmp.ensure(tb + 256));
        tb = w.tmp.cap;
        RGL_CUDA(cub::DeviceSelect::Flagged(w.tmp.p, tb, thrust::counting_iterator<uint32_t>(0), w.nz.as<uint8_t>(),
                                            w.idx.as<uint32_t>(), w.cnt.as<int>(), (int)full, st));
    }
    k_carry_chain<<<1, 1, 0, st>>>(w.cnt.as<int>(), w.idx.as<uint32_t>(), w.totals.as<float>(), w.cum.as<float>(),
                                   w.g.as<float>(), N, full);
    if (full)
        k_apply_carry<<<blocks_for(full * 8), 256, 0, st>>>(full, w.cnt.as<int>(), w.idx.as<uint32_t>(), w.cum.as<float>(),
                                                            w.g.as<float>());
    RGL_CUDA(cudaGetLastError());
    return RGL_OK;
}

int fft_forward(MomentWs& w, uint64_t M, cudaStream_t st, double2** result) {
    // ping-pong between fa and fb; input in fa
    double2* src = w.fa.as<double2>();
    double2* dst = w.fb.as<double2>();
    uint64_t Ns = 1;
    int logm = 0;
    while ((1ull << logm) < M) logm++;
    int rem = logm;
    while (rem > 0) {
        const int r = rem >= 4 ? 4 : rem;
        const uint64_t threads = M >> r;
        switch (r) {
            case 4: k_fft_pass<16><<<blocks_for(threads), 256, 0, st>>>(src, dst, M, Ns); break;
            case 3: k_fft_pass<8><<<blocks_for(threads), 256, 0, st>>>(src, dst, M, Ns); break;
            case 2: k_fft_pass<4><<<blocks_for(threads), 256, 0, st>>>(src, dst, M, Ns); break;
            default: k_fft_pass<2><<<blocks_for(threads), 256, 0, st>>>(src, dst, M, Ns); break;
        }
        Ns <<= r;
        rem -= r;
        std::swap(src, dst);
    }
    RGL_CUDA(cudaGetLastError());
    *result = src;
    return RGL_OK;
}

int dd_scan(MomentWs& w, uint64_t len, cudaStream_t st) {
    // inclusive double-double scan of w.dd_in into w.dd_out
    size_t tb = 0;
    cub::DeviceScan::InclusiveScan(nullptr, tb, w.dd_in.as<DD>(), w.dd_out.as<DD>(), DDAdd(), (int)len, st);
    RGL_TRY(w.tmp.ensure(tb + 256));
    tb = w.tmp.cap;
    RGL_CUDA(cub::DeviceScan::InclusiveScan(w.tmp.p, tb, w.dd_in.as<DD>(), w.dd_out.as<DD>(), DDAdd(), (int)len, st));
    return RGL_OK;
}

}  // namespace

namespace {
int ff_scan(MomentWs& w, uint64_t len, cudaStream_t st) {
    // inclusive float-float scan of w.dd_in (as FF) into w.dd_out
    FF* in = reinterpret_cast<FF*>(w.dd_in.p);
    FF* out = reinterpret_cast<FF*>(w.dd_out.p);
    size_t tb = 0;
    cub::DeviceScan::InclusiveScan(nullptr, tb, in, out, FFAdd(), (int)len, st);
    RGL_TRY(w.tmp.ensure(tb + 256));
    tb = w.tmp.cap;
    RGL_CUDA(cub::DeviceScan::InclusiveScan(w.tmp.p, tb, in, out, FFAdd(), (int)len, st));
    return RGL_OK;
}

// Float-float value of a long double: hi = nearest float, lo = nearest float of the remainder.
inline void ff_of(long double v, float* hi, float* lo) {
    *hi = (float)v;
    *lo = (float)(v - (long double)*hi);
}

bool g_tw16f_ready[64] = {false};

// exp(-2 pi i t / M) for t = (c << tb) (coarse table) and t < 2^tb (fine table), float-float, host-made
// in extended precision; the radix-16 constants once per device.
int ff_twiddles(MomentWs& w, uint64_t M, int device, int* tb_out) {
    if (device >= 0 && device < 64 && !g_tw16f_ready[device]) {
        float h[64];
        for (int k = 0; k < 16; k++) {
            const long double a = -2.0L * (long double)M_PI * (long double)k / 16.0L;
            ff_of(cosl(a), &h[4 * k], &h[4 * k + 1]);
            ff_of(sinl(a), &h[4 * k + 2], &h[4 * k + 3]);
        }
        RGL_CUDA(cudaMemcpyToSymbol(c_tw16f, h, sizeof(h)));
        g_tw16f_ready[device] = true;
    }
    int logm = 0;
    while ((1ull << logm) < M) logm++;
    const int tb = (logm + 1) / 2;
    const uint64_t nf = 1ull << tb, nc = (M >> tb) + 1;
    std::vector<float> h(4 * (nf + nc));
    const long double pi2 = 2.0L * 3.141592653589793238462643383279502884L;
    for (uint64_t t = 0; t < nf; t++) {
        const long double a = -pi2 * (long double)t / (long double)M;
        ff_of(cosl(a), &h[4 * t], &h[4 * t + 1]);
        ff_of(sinl(a), &h[4 * t + 2], &h[4 * t + 3]);
    }
    for (uint64_t c = 0; c < nc; c++) {
        const long double a = -pi2 * (long double)(c << tb) / (long double)M;
        float* q = &h[4 * (nf + c)];
        ff_of(cosl(a), &q[0], &q[1]);
        ff_of(sinl(a), &q[2], &q[3]);
    }
    RGL_TRY(w.grid.ensure(h.size() * 4));
    RGL_CUDA(cudaMemcpy(w.grid.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    *tb_out = tb;
    return RGL_OK;
}

int ff_fft_forward(MomentWs& w, uint64_t M, int tb, cudaStream_t st, CFF** result) {
    CFF* src = reinterpret_cast<CFF*>(w.fa.p);
    CFF* dst = reinterpret_cast<CFF*>(w.fb.p);
    const CFF* wf = reinterpret_cast<const CFF*>(w.grid.p);
    const CFF* wc = wf + (1ull << tb);
    uint64_t Ns = 1;
    int logm = 0;
    while ((1ull << logm) < M) logm++;
    int rem = logm;
    while (rem > 0) {
        const int r = rem >= 4 ? 4 : rem;
        const uint64_t threads = M >> r;
        const unsigned blocks = (unsigned)((threads + 127) / 128);
        switch (r) {
            case 4: k_ff_fft_pass<16><<<blocks, 128, 0, st>>>(src, dst, M, Ns, wc, wf, tb); break;
            case 3: k_ff_fft_pass<8><<<blocks, 128, 0, st>>>(src, dst, M, Ns, wc, wf, tb); break;
            case 2: k_ff_fft_pass<4><<<blocks, 128, 0, st>>>(src, dst, M, Ns, wc, wf, tb); break;
            default: k_ff_fft_pass<2><<<blocks, 128, 0, st>>>(src, dst, M, Ns, wc, wf, tb); break;
        }
        Ns <<= r;
        rem -= r;
        std::swap(src, dst);
    }
    RGL_CUDA(cudaGetLastError());
    *result = src;
    return RGL_OK;
}

struct GMax {
    __device__ __forceinline__ float operator()(float a, float b) const { return fmaxf(a, b); }
};

// K5-K7 of the compensated-FP32 path for the depth signal in w.g (N bins): fills outs (P0, P1, Q,
// V, UU_L, UU_R as double-double, scaled back), *uu_total, *a0 and w.gsum (as DD) for
// k_window_moments.
int moments_ff(MomentWs& w, uint64_t N, uint64_t M, int device, uint32_t G, const uint64_t* d_at, DD* outs,
               DD* uu_total, double* a0, int* scale_exp, cudaStream_t st) {
    int tb = 0;
    RGL_TRY(ff_twiddles(w, M, device, &tb));
    FF* ffin = reinterpret_cast<FF*>(w.dd_in.p);
    FF* ffout = reinterpret_cast<FF*>(w.dd_out.p);
    FF* U = reinterpret_cast<FF*>(w.U.p);
    // gsum in float-float, max(g) for the per-chromosome scale
    k_ff_from_float<<<blocks_for(N), 256, 0, st>>>(N, w.g.as<float>(), ffin);
    FF* d_gsum = reinterpret_cast<FF*>(w.gsum.p) + 4;  // beside the DD copy at w.gsum[0]
    float* d_gmax = reinterpret_cast<float*>(w.gsum.p) + 12;
    {
        size_t t1 = 0, t2 = 0;
        cub::DeviceReduce::Reduce(nullptr, t1, ffin, d_gsum, (int)N, FFAdd(), FF{0.f, 0.f}, st);
        cub::DeviceReduce::Reduce(nullptr, t2, w.g.as<float>(), d_gmax, (int)N, GMax(), 0.0f, st);
        RGL_TRY(w.tmp.ensure(std::max(t1, t2) + 256));
        t1 = w.tmp.cap;
        RGL_CUDA(cub::DeviceReduce::Reduce(w.tmp.p, t1, ffin, d_gsum, (int)N, FFAdd(), FF{0.f, 0.f}, st));
        t2 = w.tmp.cap;
        RGL_CUDA(cub::DeviceReduce::Reduce(w.tmp.p, t2, w.g.as<float>(), d_gmax, (int)N, GMax(), 0.0f, st));
    }
    FF gs;
    float gmax = 0.f;
    RGL_CUDA(cudaMemcpyAsync(&gs, d_gsum, sizeof(FF), cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaMemcpyAsync(&gmax, d_gmax, 4, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    // the DD copy of the sum for the final reduction (exact: hi + lo of a float-float)
    const DD gsum_dd{(double)gs.hi + (double)gs.lo, 0.0};
    RGL_CUDA(cudaMemcpyAsync(w.gsum.p, &gsum_dd, sizeof(DD), cudaMemcpyHostToDevice, st));
    // |u| <= max(g) (coverage is non-negative): scale u by 2^-e with 2^e >= max(g)
    int e = 0;
    if (gmax > 0.f) (void)std::frexp((double)gmax, &e);
    const float scale = std::ldexp(1.0f, -e);
    *scale_exp = e;
    k_ff_center<<<blocks_for(M), 256, 0, st>>>(N, M, w.g.as<float>(), d_gsum, scale, reinterpret_cast<CFF*>(w.fa.p),
                                                ffin);
    RGL_TRY(ff_scan(w, N + 1, st));
    k_ff_shift<<<blocks_for(N + 1), 256, 0, st>>>(N, ffout, U);
    CFF* X = nullptr;
    RGL_TRY(ff_fft_forward(w, M, tb, st, &X));
    k_ff_power<<<blocks_for(M), 256, 0, st>>>(M, X);
    if (X != reinterpret_cast<CFF*>(w.fa.p)) RGL_CUDA(cudaMemcpyAsync(w.fa.p, X, M * 16, cudaMemcpyDeviceToDevice, st));
    CFF* Y = nullptr;
    RGL_TRY(ff_fft_forward(w, M, tb, st, &Y));
    const float inv_m = std::ldexp(1.0f, -(int)std::lround(std::log2((double)M)));
    const int terms[4] = {T_A, T_MA, T_U2, T_V2};
    for (int q = 0; q < 4; q++) {
        k_ff_term<<<blocks_for(N + 1), 256, 0, st>>>(N + 1, terms[q], Y, inv_m, U, N, ffin);
        RGL_TRY(ff_scan(w, N + 1, st));
        k_ff_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at, ffout, 2 * e, outs + (uint64_t)q * G);
    }
    k_ff_term<<<blocks_for(N + 1), 256, 0, st>>>(N + 1, T_U, Y, inv_m, U, N, ffin);
    RGL_TRY(ff_scan(w, N + 1, st));
    k_ff_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at, ffout, e, outs + 4ull * G);
    k_ff_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at + G, ffout, e, outs + 5ull * G);
    FF tot, y0;
    RGL_CUDA(cudaMemcpyAsync(&tot, ffout + N, sizeof(FF), cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaMemcpyAsync(&y0, &Y[0].re, sizeof(FF), cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    *uu_total = DD{std::ldexp((double)tot.hi, e), std::ldexp((double)tot.lo, e)};
    *a0 = std::ldexp(((double)y0.hi + (double)y0.lo) * (double)inv_m, 2 * e);
    RGL_CUDA(cudaGetLastError());
    return RGL_OK;
}

}  // namespace

struct rgl_moments;  // defined in stats.cu
namespace rgl {
int moments_table_ptr(rgl_moments* m, uint32_t sid, uint32_t chrom, float2** ptr, uint64_t* slots, uint64_t* n_bins,
                      int* device);
int moments_mark(rgl_moments* m, uint32_t sid, uint32_t chrom, uint64_t entries);
}  // namespace rgl

extern "C" {

int rgl_depth_signal(int device, const rgl_interval* intervals, uint64_t n, uint64_t n_bins, uint32_t bin_size,
                     float* g_out) {
    clear_error();
    if ((n && !intervals) || !g_out || bin_size == 0) return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    if (n_bins * (uint64_t)bin_size > 0xFFFFFFFFull) return fail(RGL_ERR_INVALID_ARGUMENT, "n_bins * bin_size overflows u32");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RGL_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= 16 || device >= ndev) return fail(RGL_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    DeviceScope scope;
    RGL_TRY(scope.enter(device));
    std::lock_guard<std::mutex> lk(g_ws_mu);
    RGL_TRY(depth_signal_dev(g_ws[device], intervals, n, n_bins, bin_size, 0));
    RGL_CUDA(cudaMemcpy(g_out, g_ws[device].g.p, n_bins * 4, cudaMemcpyDeviceToHost));
    return RGL_OK;
}

int rgl_moments_build_ex(rgl_moments* m, uint32_t sid, uint32_t chrom, const rgl_interval* intervals, uint64_t n,
                         uint32_t bin_size, uint32_t precision, double* mean_out, double* var_out) {
    clear_error();
    if (!m || (n && !intervals) || bin_size == 0) return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    if (precision != RGL_MOM_FP64 && precision != RGL_MOM_FP32C)
        return fail(RGL_ERR_INVALID_ARGUMENT, "precision must be RGL_MOM_FP64 or RGL_MOM_FP32C");
    float2* table = nullptr;
    uint64_t slots = 0, N = 0;
    int device = 0;
    RGL_TRY(moments_table_ptr(m, sid, chrom, &table, &slots, &N, &device));
    if (N * (uint64_t)bin_size > 0xFFFFFFFFull) return fail(RGL_ERR_INVALID_ARGUMENT, "n_bins * bin_size overflows u32");
    if (device < 0 || device >= 16) return fail(RGL_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    if (N <= 1) return moments_mark(m, sid, chrom, 0);  // moments_from_signal returns no entries
    if (N >= (1ull << 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 bins per chromosome");
    DeviceScope scope;
    RGL_TRY(scope.enter(device));
    std::lock_guard<std::mutex> lk(g_ws_mu);
    MomentWs& w = g_ws[device];
    cudaStream_t st = 0;
    RGL_TRY(upload_twiddles(device));
    RGL_TRY(depth_signal_dev(w, intervals, n, N, bin_size, st));
    uint64_t M = 1;
    while (M < 2 * N) M <<= 1;
    RGL_TRY(w.fa.ensure(M * 16));
    RGL_TRY(w.fb.ensure(M * 16));
    RGL_TRY(w.dd_in.ensure((N + 2) * 16));
    RGL_TRY(w.dd_out.ensure((N + 2) * 16));
    RGL_TRY(w.U.ensure((N + 2) * 8));
    RGL_TRY(w.gsum.ensure(64));
    // K7 gather points: the L grid of the store
    const std::vector<uint64_t> grid = moment_grid(N);
    const uint32_t G = (uint32_t)grid.size();
    if (G != slots) return fail(RGL_ERR_INVALID_ARGUMENT, "moment table size does not match the L grid");
    std::vector<uint64_t> at_l(G), at_r(G);
    for (uint32_t i = 0; i < G; i++) {
        at_l[i] = grid[i] - 1;  // inclusive prefix over t < L (the t = 0 term of P0 / P1 is zero)
        at_r[i] = N - grid[i];  // UU(N-L+1) = sum_{s<=N-L} U[s]
    }
    RGL_TRY(w.at.ensure(G * 8 * 3ull + 64));
    RGL_TRY(w.gl.ensure(G * 8ull + 64));
    RGL_TRY(w.outs.ensure(G * 16 * 7ull + 64));
    uint64_t* d_at = w.at.as<uint64_t>();
    RGL_CUDA(cudaMemcpyAsync(d_at, at_l.data(), G * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(d_at + G, at_r.data(), G * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(w.gl.p, grid.data(), G * 8, cudaMemcpyHostToDevice, st));
    DD* outs = w.outs.as<DD>();  // P0, P1, Q, V, UU_L, UU_R (G each)
    DD uu_total{0.0, 0.0};
    double a0 = 0.0;
    int ff_exp = 0;
    if (precision == RGL_MOM_FP32C) {
        RGL_TRY(moments_ff(w, N, M, device, G, d_at, outs, &uu_total, &a0, &ff_exp, st));
    } else {
        // K5: mean of g (double-double sum), centred signal, U = prefix of u
        k_to_dd<<<blocks_for(N), 256, 0, st>>>(N, w.g.as<float>(), w.dd_in.as<DD>());
        {
            size_t tb = 0;
            cub::DeviceReduce::Reduce(nullptr, tb, w.dd_in.as<DD>(), w.gsum.as<DD>(), (int)N, DDAdd(), DD{0.0, 0.0}, st);
            RGL_TRY(w.tmp.ensure(tb + 256));
            tb = w.tmp.cap;
            RGL_CUDA(cub::DeviceReduce::Reduce(w.tmp.p, tb, w.dd_in.as<DD>(), w.gsum.as<DD>(), (int)N, DDAdd(),
                                               DD{0.0, 0.0}, st));
        }
        k_center<<<blocks_for(M), 256, 0, st>>>(N, M, w.g.as<float>(), w.gsum.as<DD>(), w.fa.as<double2>(),
                                                 w.dd_in.as<DD>());
        // exclusive prefix: U[s] = sum_{k<s} u[k] for s = 0..N -> inclusive scan of u shifted by one
        RGL_TRY(dd_scan(w, N + 1, st));  // dd_out[s] = sum_{k<=s} u[k]
        RGL_CUDA(cudaMemsetAsync(w.U.p, 0, 8, st));
        k_dd_to_double<<<blocks_for(N), 256, 0, st>>>(N, w.dd_out.as<DD>(), w.U.as<double>() + 1);
        // K6: A[m] = Re(FFT(|FFT(u)|^2))[m] / M
        double2* X = nullptr;
        RGL_TRY(fft_forward(w, M, st, &X));
        k_power<<<blocks_for(M), 256, 0, st>>>(M, X);
        if (X != w.fa.as<double2>()) RGL_CUDA(cudaMemcpyAsync(w.fa.p, X, M * 16, cudaMemcpyDeviceToDevice, st));
        double2* Y = nullptr;
        RGL_TRY(fft_forward(w, M, st, &Y));
        // K7: prefix sums at the grid points
        const double inv_m = 1.0 / (double)M;
        const int terms[4] = {T_A, T_MA, T_U2, T_V2};
        for (int q = 0; q < 4; q++) {
            k_term<<<blocks_for(N + 1), 256, 0, st>>>(N + 1, terms[q], Y, inv_m, w.U.as<double>(), N, w.dd_in.as<DD>());
            RGL_TRY(dd_scan(w, N + 1, st));
            k_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at, w.dd_out.as<DD>(), outs + (uint64_t)q * G);
        }
        k_term<<<blocks_for(N + 1), 256, 0, st>>>(N + 1, T_U, Y, inv_m, w.U.as<double>(), N, w.dd_in.as<DD>());
        RGL_TRY(dd_scan(w, N + 1, st));
        // UU(L) = sum_{s<L} U[s] = inclusive[L-1]; UU(N-L+1) = inclusive[N-L]; UU(N+1) = inclusive[N]
        k_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at, w.dd_out.as<DD>(), outs + 4ull * G);
        k_gather<<<blocks_for(G), 256, 0, st>>>(G, d_at + G, w.dd_out.as<DD>(), outs + 5ull * G);
        double2 a0c;
        RGL_CUDA(cudaMemcpyAsync(&uu_total, w.dd_out.as<DD>() + N, sizeof(DD), cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(&a0c, Y, sizeof(double2), cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaStreamSynchronize(st));
        a0 = a0c.x * inv_m;
    }
    // the final reduction and the variance subtraction, FP64 (both paths)
    DevBuf& dm = w.mv;
    RGL_TRY(dm.ensure(G * 16ull + 64));
    double* d_mean = mean_out ? dm.as<double>() : nullptr;
    double* d_var = var_out ? dm.as<double>() + G : nullptr;
    // windows with few positions: the variance reduced directly from the prefix sums (k_direct_var)
    const uint64_t few = std::max<uint64_t>(65536, N / 32);
    std::vector<uint32_t> direct;
    for (uint32_t i = 0; i < G; i++)
        if (N - grid[i] + 1 <= few) direct.push_back(i);
    RGL_TRY(w.dv.ensure(G * 8ull + 64));
    RGL_CUDA(cudaMemsetAsync(w.dv.p, 0xFF, G * 8ull, st));  // NaN: not reduced directly
    if (!direct.empty()) {
        uint32_t* d_which = reinterpret_cast<uint32_t*>(d_at + 2ull * G);
        RGL_CUDA(cudaMemcpyAsync(d_which, direct.data(), direct.size() * 4, cudaMemcpyHostToDevice, st));
        if (precision == RGL_MOM_FP32C)
            k_direct_var<FF><<<(unsigned)direct.size(), 256, 0, st>>>(
                d_which, w.gl.as<uint64_t>(), N, reinterpret_cast<const FF*>(w.U.p), std::ldexp(1.0, ff_exp),
                w.dv.as<double>());
        else
            k_direct_var<double><<<(unsigned)direct.size(), 256, 0, st>>>(d_which, w.gl.as<uint64_t>(), N,
                                                                           w.U.as<double>(), 1.0, w.dv.as<double>());
    }
    k_window_moments<<<blocks_for(G), 256, 0, st>>>(G, w.gl.as<uint64_t>(), N, w.gsum.as<DD>(), a0, outs, outs + G,
                                                    outs + 2ull * G, outs + 3ull * G, outs + 4ull * G, outs + 5ull * G,
                                                    uu_total, table, d_mean, d_var, w.dv.as<double>());
    RGL_CUDA(cudaGetLastError());
    if (mean_out) RGL_CUDA(cudaMemcpyAsync(mean_out, d_mean, G * 8, cudaMemcpyDeviceToHost, st));
    if (var_out) RGL_CUDA(cudaMemcpyAsync(var_out, d_var, G * 8, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    return moments_mark(m, sid, chrom, G);
}

int rgl_moments_build(rgl_moments* m, uint32_t sid, uint32_t chrom, const rgl_interval* intervals, uint64_t n,
                      uint32_t bin_size, double* mean_out, double* var_out) {
    return rgl_moments_build_ex(m, sid, chrom, intervals, n, bin_size, RGL_MOM_FP64, mean_out, var_out);
}

}  // extern "C"

// ================================================================================================
// Allocation-free depth signal.
//
// Some callers cannot allocate device memory while they call this library: code that is recording
// a CUDA graph (cudaMalloc / cudaFree are not capturable operations), hosts that route every
// device allocation through their own arena or memory pool and forbid allocations behind its back,
// and latency-critical loops that cannot afford cudaMalloc's implicit device-wide synchronisation.
// rgl_depth_signal_noalloc serves them: the same bit-exact depth signal as rgl_depth_signal, from
// device-resident intervals into a caller-provided device buffer, with all of its scratch (impulse
// records, sort buffers, per-chunk carries, CUB temporary storage) in one fixed array in this
// file.  The array is a static device variable: every GPU that loads the library holds its
// RGL_NOALLOC_SCRATCH_BYTES until the process exits.
// ================================================================================================
namespace {

constexpr uint64_t kNaMaxIv = RGL_NOALLOC_MAX_INTERVALS;
constexpr uint64_t kNaMaxBins = RGL_NOALLOC_MAX_BINS;
constexpr uint64_t kNaKeys = 4 * kNaMaxIv * 8;           // one key array (u64 x 4 records per interval)
constexpr uint64_t kNaVals = 4 * kNaMaxIv * 4;           // one value array (f32)
constexpr uint64_t kNaChunks = kNaMaxBins / 8;
constexpr uint64_t kNaOffKeyA = 0;
constexpr uint64_t kNaOffKeyB = kNaOffKeyA + kNaKeys;
constexpr uint64_t kNaOffValA = kNaOffKeyB + kNaKeys;
constexpr uint64_t kNaOffValB = kNaOffValA + kNaVals;
constexpr uint64_t kNaOffTot = kNaOffValB + kNaVals;
constexpr uint64_t kNaOffIdx = kNaOffTot + kNaChunks * 4;
constexpr uint64_t kNaOffCum = kNaOffIdx + kNaChunks * 4;
constexpr uint64_t kNaOffNz = kNaOffCum + kNaChunks * 4;
constexpr uint64_t kNaOffCnt = kNaOffNz + ((kNaChunks + 255) / 256) * 256;
constexpr uint64_t kNaOffTmp = kNaOffCnt + 256;
static_assert(kNaOffTmp < RGL_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds its array");
constexpr uint64_t kNaTmpBytes = RGL_NOALLOC_SCRATCH_BYTES - kNaOffTmp;

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[RGL_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_na_mu;
struct NoallocSlot {
    unsigned long long ctx_id = 0;  // the context the address belongs to (0: not looked up yet)
    unsigned char* ptr = nullptr;   // device address of g_noalloc_scratch in that context
};
NoallocSlot g_na[64];

// The unique id of the calling thread's current context (cuCtxGetId, unique for the life of the
// process, so a context destroyed by cudaDeviceReset and made again gets a new one), through the
// runtime's driver entry points so that the library needs no link against libcuda.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
int current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess || !f1 || !f2)
            return fail(RGL_ERR_DEVICE, "driver entry points cuCtxGetCurrent / cuCtxGetId are unavailable");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx) return fail(RGL_ERR_DEVICE, "no current CUDA context");
    if (get_id(ctx, id) != 0) return fail(RGL_ERR_DEVICE, "cuCtxGetId failed");
    return RGL_OK;
}

// With `device` current: the array's device address in the current context (the symbol itself is
// only a host-side stand-in), looked up on the first call and again whenever the device's context
// has changed since (after cudaDeviceReset the module is loaded anew, possibly elsewhere), and a
// check that CUB's temporary storage for the largest inputs fits.
int noalloc_setup(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    unsigned long long id = 0;
    RGL_TRY(current_context_id(&id));
    NoallocSlot& slot = g_na[device];
    if (slot.ctx_id != id || !slot.ptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(RGL_ERR_DEVICE, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        size_t sort_b = 0, sel_b = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, sort_b, (uint64_t*)nullptr, (uint64_t*)nullptr, (float*)nullptr,
                                        (float*)nullptr, (int)(4 * kNaMaxIv), 0, 64);
        cub::DeviceSelect::Flagged(nullptr, sel_b, thrust::counting_iterator<uint32_t>(0), (uint8_t*)nullptr,
                                   (uint32_t*)nullptr, (int*)nullptr, (int)kNaChunks);
        if (std::max(sort_b, sel_b) > kNaTmpBytes)
            return fail(RGL_ERR_UNSUPPORTED, "CUB temporary storage exceeds the reserved scratch");
        slot.ptr = static_cast<unsigned char*>(p);
        slot.ctx_id = id;
    }
    *out = slot.ptr;
    return RGL_OK;
}
}  // namespace

extern "C" int rgl_depth_signal_noalloc(int device, const rgl_interval* d_intervals, uint64_t n, uint64_t n_bins,
                                        uint32_t bin_size, float* d_g, void* stream) {
    clear_error();
    if ((n && !d_intervals) || !d_g || bin_size == 0 || n_bins == 0) return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    if (n > kNaMaxIv)
        return fail(RGL_ERR_INVALID_ARGUMENT, "rgl_depth_signal_noalloc takes at most " +
                                                  std::to_string(kNaMaxIv) + " intervals (got " + std::to_string(n) + ")");
    if (n_bins > kNaMaxBins)
        return fail(RGL_ERR_INVALID_ARGUMENT, "rgl_depth_signal_noalloc takes at most " +
                                                  std::to_string(kNaMaxBins) + " bins (got " + std::to_string(n_bins) + ")");
    if (n_bins * (uint64_t)bin_size > 0xFFFFFFFFull) return fail(RGL_ERR_INVALID_ARGUMENT, "n_bins * bin_size overflows u32");
    // the chunk pass reads and writes d_g as float4, the spike pass reads the intervals as u32 words
    if (reinterpret_cast<uintptr_t>(d_g) % 16 != 0)
        return fail(RGL_ERR_INVALID_ARGUMENT, "d_g must be 16-byte aligned");
    if (reinterpret_cast<uintptr_t>(d_intervals) % 4 != 0)
        return fail(RGL_ERR_INVALID_ARGUMENT, "d_intervals must be 4-byte aligned");
    if (device < 0 || device >= 64) return fail(RGL_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    DeviceScope scope;
    RGL_TRY(scope.enter(device));
    unsigned char* base = nullptr;
    RGL_TRY(noalloc_setup(device, &base));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint64_t* key_a = reinterpret_cast<uint64_t*>(base + kNaOffKeyA);
    uint64_t* key_b = reinterpret_cast<uint64_t*>(base + kNaOffKeyB);
    float* val_a = reinterpret_cast<float*>(base + kNaOffValA);
    float* val_b = reinterpret_cast<float*>(base + kNaOffValB);
    float* totals = reinterpret_cast<float*>(base + kNaOffTot);
    uint32_t* idx = reinterpret_cast<uint32_t*>(base + kNaOffIdx);
    float* cum = reinterpret_cast<float*>(base + kNaOffCum);
    uint8_t* nz = base + kNaOffNz;
    int* cnt = reinterpret_cast<int*>(base + kNaOffCnt);
    void* tmp = base + kNaOffTmp;
    // the output and the compacted-chunk count start at zero; every other scratch word a call reads
    // it writes first
    RGL_CUDA(cudaMemsetAsync(d_g, 0, n_bins * 4, st));
    RGL_CUDA(cudaMemsetAsync(cnt, 0, 4, st));
    if (n) {
        const uint64_t m = 4 * n;
        k_spike_records<<<blocks_for(n), 256, 0, st>>>((uint32_t)n, d_intervals, (uint32_t)n_bins, bin_size, key_a, val_a);
        size_t tb = kNaTmpBytes;
        RGL_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key_a, key_b, val_a, val_b, (int)m, 0, 64, st));
        k_bin_sums<<<blocks_for(m), 256, 0, st>>>(m, key_b, val_b, d_g);
    }
    if (n_bins > 1) {
        const uint64_t full = n_bins / 8;
        if (full) {
            k_chunk_local<<<blocks_for(full), 256, 0, st>>>(full, d_g, totals, nz);
            size_t tb = kNaTmpBytes;
            RGL_CUDA(cub::DeviceSelect::Flagged(tmp, tb, thrust::counting_iterator<uint32_t>(0), nz, idx, cnt,
                                                (int)full, st));
        }
        k_carry_chain<<<1, 1, 0, st>>>(cnt, idx, totals, cum, d_g, n_bins, full);
        if (full) k_apply_carry<<<blocks_for(full * 8), 256, 0, st>>>(full, cnt, idx, cum, d_g);
    }
    RGL_CUDA(cudaGetLastError());
    return RGL_OK;
}

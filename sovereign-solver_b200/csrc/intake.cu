// intake.cu -- problem intake on the device: row binning and Ruiz +
// Pock-Chambolle scaling (Scaling::equilibrate, src/l1/scaling.cpp:19-104 and
// :155-205) without a host pass over the matrix.
//
// The factors are bit-identical to the reference's host computation:
//   * Ruiz row/column maxima of |a| * r_i * c_j are order-free (max), each
//     product formed as (|a| * r_i) * c_j like scaling.cpp:48-50;
//   * the update r_i /= sqrt(max) uses IEEE sqrt and division;
//   * Pock-Chambolle sums are added per row (per A^T row for the columns) in
//     the reference's order (CSR order for rows, ascending row for columns,
//     scaling.cpp:85-96), by one thread or, for long rows, one warp that adds
//     in the same order (ordered.cuh); with alpha = 1 the exponents are 1 and the
//     term is the magnitude itself (pow(m, 1) == m exactly), other alphas call
//     the device pow;
//   * the early exit of the Ruiz sweeps (worst < tolerance) is decided by the
//     last CTA of each update and read by the next sweep's kernels.
#include <algorithm>
#include <cmath>

#include "engine.cuh"
#include "ordered.cuh"

namespace pdhg {

namespace {

__host__ __device__ inline int nblocks(int64_t n) {
    return static_cast<int>((n + kBlock - 1) / kBlock);
}

__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ bool fb(double v) { return v > -INFINITY && v < INFINITY; }
__device__ __forceinline__ double safe_sqrt(double v) { return v > 0.0 ? sqrt(v) : 1.0; }

__device__ __forceinline__ bool last_cta(unsigned int* ticket) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    return am_last;
}

__device__ __forceinline__ unsigned group_mask(int vw) {
    if (vw >= 32) return 0xffffffffu;
    const unsigned base = (threadIdx.x & 31u) & ~static_cast<unsigned>(vw - 1);
    return ((1u << vw) - 1u) << base;
}

// Problem checks of Problem::validate (src/io/problem.cpp:50-) and
// CsrMatrix::validate (src/l0/sparse.cpp:94-128) as flags: bit 0 a column
// (non-finite cost, NaN or crossed bounds), bit 1 a row (NaN or crossed
// bounds), bit 2 an entry's column out of range, bit 3 an entry not strictly
// ascending in its row or with a non-finite value. row_ptr itself must already be known monotone and
// within [0, nnz]. Which item fails first, and the message, is left to the
// host check, which only runs when a flag is set. Entries are checked by
// groups of `lanes` threads per row. c == NULL skips the column checks,
// rlo == NULL the row checks (a matrix on its own).
__global__ void __launch_bounds__(kBlock) k_validate(int32_t m, int32_t n, const int32_t* rp,
                                                     const int32_t* ci, const double* v,
                                                     const double* c, const double* clo,
                                                     const double* chi, const double* rlo,
                                                     const double* rhi, int lanes,
                                                     unsigned* flags) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kBlock;
    const int64_t t0 = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    unsigned bad = 0;
    for (int64_t j = t0; c != nullptr && j < n; j += stride) {
        const double lo = clo[j], hi = chi[j];
        if (!isfinite(c[j]) || isnan(lo) || isnan(hi) || lo > hi) bad |= 1u;
    }
    for (int64_t i = t0; rlo != nullptr && i < m; i += stride) {
        const double lo = rlo[i], hi = rhi[i];
        if (isnan(lo) || isnan(hi) || lo > hi) bad |= 2u;
    }
    const int64_t groups = static_cast<int64_t>(m) * lanes;
    for (int64_t g = t0; g < groups; g += stride) {
        const int64_t r = g / lanes;
        const int b = rp[r], e = rp[r + 1];
        for (int k = b + static_cast<int>(g % lanes); k < e; k += lanes) {
            const int col = ci[k];
            if (col < 0 || col >= n) bad |= 4u;
            if ((k > b && ci[k - 1] >= col) || !isfinite(v[k])) bad |= 8u;
        }
    }
    for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(flags, bad);
}

// Row lengths -> long-row list, number and total length of short rows
// (grid-stride, one atomic per CTA and counter).
// *flag |= 1 when some row's length differs from row 0's (grid-stride).
__global__ void k_uniform_rows(const int32_t* rp, int32_t rows, unsigned* flag) {
    const int len0 = rp[1] - rp[0];
    bool diff = false;
    for (int64_t r = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; r < rows;
         r += static_cast<int64_t>(gridDim.x) * kBlock)
        diff = diff || (rp[r + 1] - rp[r] != len0);
    if (diff) atomicOr(flag, 1u);
}

// *flag |= 1 when some entry differs from entry 0 (grid-stride; +-inf compare
// equal to themselves).
__global__ void k_uniform_vec(const double* v, int32_t n, unsigned* flag) {
    const double v0 = v[0];
    bool diff = false;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; t < n;
         t += static_cast<int64_t>(gridDim.x) * kBlock)
        diff = diff || !(v[t] == v0);
    if (diff) atomicOr(flag, 1u);
}

__global__ void k_bin(const int32_t* rp, int32_t rows, int long_threshold, int32_t* long_rows,
                      unsigned long long* counters) {
    unsigned long long ns = 0, nz = 0;
    for (int64_t r = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; r < rows;
         r += static_cast<int64_t>(gridDim.x) * kBlock) {
        const int len = rp[r + 1] - rp[r];
        if (len > long_threshold) {
            const unsigned long long slot = atomicAdd(&counters[0], 1ull);
            long_rows[slot] = static_cast<int32_t>(r);
        } else {
            ns += 1;
            nz += static_cast<unsigned long long>(len);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ns += __shfl_xor_sync(0xffffffffu, ns, o);
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    __shared__ unsigned long long sh[2][kBlock / 32];
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = ns;
        sh[1][threadIdx.x >> 5] = nz;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        unsigned long long t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += sh[threadIdx.x][w];
        if (t) atomicAdd(&counters[1 + threadIdx.x], t);
    }
}

__global__ void k_row_extents(const int32_t* rows, int32_t n, const int32_t* rp, int4* out) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= n) return;
    const int32_t r = rows[k];
    out[k] = make_int4(r, rp[r], rp[r + 1], 0);
}

__global__ void k_gather_cols(const int32_t* ci, const int64_t* pos, int32_t n, int32_t* out) {
    const int q = blockIdx.x * kBlock + threadIdx.x;
    if (q < n) out[q] = ci[pos[q]];
}

// One CTA per slice (grid-stride over slices): entry k of lane l from the
// CSR row S.row[32 s + l], or padding (column 0, value 0) past the row's end.
__global__ void k_fill_slices(const int32_t* rp, const int32_t* ci, const double* v64,
                              const float* v32, RowSlices S, int32_t* col, float* o32,
                              double* o64) {
    for (int sl = blockIdx.x; sl < S.n_slice; sl += gridDim.x) {
        const int4 d = S.slice[sl];
        const int64_t n = static_cast<int64_t>(d.x) * 32;
        for (int64_t e = threadIdx.x; e < n; e += kBlock) {
            const int l = static_cast<int>(e & 31);
            const int k = static_cast<int>(e >> 5);
            const int r = S.row[32 * sl + l];
            const int64_t dst = d.y + e;
            if (r >= 0 && k < S.rlen[32 * sl + l]) {
                const int64_t src = rp[r] + k;
                col[dst] = ci[src];
                o32[dst] = v32[src];
                o64[dst] = v64[src];
            } else {
                col[dst] = 0;
                o32[dst] = 0.f;
                o64[dst] = 0.0;
            }
        }
    }
}

// Affine slices: where every entry of a slice (lane l, step k, k below the
// lane's row length) is column base + l + k * stride, the slice kernel
// computes the columns instead of loading them. {base, stride}, or {0, 0} for
// a slice with any other entry; every entry is compared.
__global__ void k_affine_slices(RowSlices S, int2* affine, unsigned long long* nnz_affine) {
    __shared__ int ok;
    for (int sl = blockIdx.x; sl < S.n_slice; sl += gridDim.x) {
        const int4 d = S.slice[sl];
        const int64_t base = S.col[d.y];
        const int64_t stride = d.x > 1 ? static_cast<int64_t>(S.col[d.y + 32]) - base : 0;
        if (threadIdx.x == 0) ok = stride > 0 ? 1 : 0;
        __syncthreads();
        const int64_t n = static_cast<int64_t>(d.x) * 32;
        bool bad = false;
        for (int64_t e = threadIdx.x; e < n; e += kBlock) {
            const int l = static_cast<int>(e & 31);
            const int k = static_cast<int>(e >> 5);
            if (k < S.rlen[32 * sl + l] && S.col[d.y + e] != base + l + k * stride) bad = true;
        }
        if (bad) ok = 0;  // every writer writes 0
        __syncthreads();
        if (threadIdx.x == 0) {
            affine[sl] = ok ? make_int2(static_cast<int>(base), static_cast<int>(stride)) : make_int2(0, 0);
            if (ok) {
                unsigned long long len = 0;
                for (int l = 0; l < 32; ++l) len += static_cast<unsigned long long>(S.rlen[32 * sl + l]);
                atomicAdd(nnz_affine, len);
            }
        }
        __syncthreads();
    }
}

// Dense rows: a long row whose entries k = b..e-1 sit in columns k + off
// (consecutive columns, a supply row of a transportation LP) gets off in
// dense_off[row], so the iteration kernels compute the columns instead of
// loading them and stream the gathered vector. Every entry is compared; the
// other rows keep kNotDense (set before the launch).
__global__ void k_dense_rows(const int32_t* ci, const int4* ext, int32_t n_ext, int32_t* dense_off,
                             unsigned long long* nnz_dense) {
    __shared__ int ok;
    for (int q = blockIdx.x; q < n_ext; q += gridDim.x) {
        const int4 w = ext[q];
        const int off = ci[w.y] - w.y;
        if (threadIdx.x == 0) ok = off != kNotDense ? 1 : 0;
        __syncthreads();
        bool bad = false;
        for (int k = w.y + static_cast<int>(threadIdx.x); k < w.z; k += kBlock)
            if (ci[k] - k != off) bad = true;
        if (bad) ok = 0;  // every writer writes 0
        __syncthreads();
        if (threadIdx.x == 0 && ok) {
            dense_off[w.x] = off;
            atomicAdd(nnz_dense, static_cast<unsigned long long>(w.z - w.y));
        }
        __syncthreads();
    }
}

// Rows with lo < length <= hi appended to `list` (grid-stride; one atomic per
// warp that has any).
__global__ void k_bin_range(const int32_t* rp, int32_t rows, int lo, int hi, int32_t* list,
                            unsigned long long* count) {
    for (int64_t r0 = blockIdx.x * static_cast<int64_t>(kBlock); r0 < rows;
         r0 += static_cast<int64_t>(gridDim.x) * kBlock) {
        const int64_t r = r0 + threadIdx.x;
        bool in = false;
        if (r < rows) {
            const int len = rp[r + 1] - rp[r];
            in = len > lo && len <= hi;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, in);
        if (mask == 0u) continue;
        const int lane = threadIdx.x & 31;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(count, static_cast<unsigned long long>(__popc(mask)));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (in) list[base + __popc(mask & ((1u << lane) - 1u))] = static_cast<int32_t>(r);
    }
}

// (|v| * rs_i) * cs_j for entry k of row r (transposed: the row is column j).
__device__ __forceinline__ double scaled_mag(const DevCsr& M, int transposed, const double* rs,
                                             const double* cs, int r, int k) {
    const int c = M.ci[k];
    return transposed ? fabs(M.v64[k]) * rs[c] * cs[r] : fabs(M.v64[k]) * rs[r] * cs[c];
}

// Ruiz maxima of one orientation (order-free): short rows by groups of M.vw
// lanes, long rows by one CTA each, as in the iteration kernels.
__global__ void __launch_bounds__(kBlock) k_ruiz_max(DevCsr M, int transposed, const double* rs,
                                                     const double* cs, const IntakeState* is,
                                                     double* out, int short_blocks) {
    if (is->ruiz_done) return;
    if (static_cast<int>(blockIdx.x) < short_blocks) {
        const int vw = M.vw;
        const int lane = threadIdx.x & (vw - 1);
        const int r = (blockIdx.x * kBlock + threadIdx.x) / vw;
        if (r >= M.rows) return;
        const int b = M.rp[r], e = M.rp[r + 1];
        if (e - b > kLongRow) return;
        double mx = 0.0;
        for (int k = b + lane; k < e; k += vw) mx = smax(mx, scaled_mag(M, transposed, rs, cs, r, k));
        const unsigned mask = group_mask(vw);
        for (int o = vw / 2; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(mask, mx, o));
        if (lane == 0) out[r] = mx;
    } else {
        const int r = M.long_rows[blockIdx.x - short_blocks];
        double mx = 0.0;
        for (int k = M.rp[r] + threadIdx.x; k < M.rp[r + 1]; k += kBlock)
            mx = smax(mx, scaled_mag(M, transposed, rs, cs, r, k));
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        __shared__ double sh[kBlock / 32];
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kBlock / 32; ++w) t = fmax(t, sh[w]);
            out[r] = t;
        }
    }
}

__global__ void k_ruiz_update(int32_t m, int32_t n, double* rs, double* cs,
                              const double* row_max, const double* col_max, double tol,
                              IntakeState* is) {
    if (is->ruiz_done) return;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    double worst = 0.0;
    if (t < m && row_max[t] > 0.0) {
        rs[t] /= safe_sqrt(row_max[t]);
        worst = fabs(row_max[t] - 1.0);
    }
    if (t < n && col_max[t] > 0.0) {
        cs[t] /= safe_sqrt(col_max[t]);
        worst = smax(worst, fabs(col_max[t] - 1.0));
    }
    for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    __shared__ double shw[kBlock / 32];
    if ((threadIdx.x & 31) == 0) shw[threadIdx.x >> 5] = worst;
    __syncthreads();
    if (threadIdx.x == 0) {
        double w = 0.0;
        for (int i = 0; i < kBlock / 32; ++i) w = fmax(w, shw[i]);
        if (w > 0.0) atomicMax(&is->worst, static_cast<unsigned long long>(__double_as_longlong(w)));
    }
    if (!last_cta(&is->ticket) || threadIdx.x != 0) return;
    const double w = __longlong_as_double(static_cast<long long>(
        *reinterpret_cast<volatile unsigned long long*>(&is->worst)));
    if (w < tol) is->ruiz_done = 1;  // scaling.cpp:72
    is->worst = 0ull;
    is->ticket = 0u;
}

__device__ __forceinline__ double pc_term(double mag, double e) {
    return e == 1.0 ? mag : pow(mag, e);
}

// Pock-Chambolle sums, one thread per row, in the reference's order; the
// loads of four entries are issued before their terms are added.
// Skipped entries (magnitude 0) are added as +0.0 in the warp path: the sum
// starts at +0.0 and every term is >= +0.0, so adding +0.0 changes no bit.
__global__ void __launch_bounds__(kBlock) k_pc_sum(DevCsr M, int transposed, const double* rs,
                                                   const double* cs, double expo, double* out) {
    const RowTask t = row_task(M, blockIdx.x);
    if (t.row < 0) return;
    const int r = t.row;
    const int b = M.rp[r], e = M.rp[r + 1];
    double sum = 0.0;
    if (t.warp) {
        sum = ordered_sum_warp(
            b, e,
            [&](int k) {
                const double mag = scaled_mag(M, transposed, rs, cs, r, k);
                return mag > 0.0 ? pc_term(mag, expo) : 0.0;
            },
            0.0, warp_stage());
    } else {
        int k = b;
        for (; k + 4 <= e; k += 4) {
            double mg[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) mg[u] = scaled_mag(M, transposed, rs, cs, r, k + u);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (mg[u] > 0.0) sum = __dadd_rn(sum, pc_term(mg[u], expo));
        }
        for (; k < e; ++k) {
            const double mag = scaled_mag(M, transposed, rs, cs, r, k);
            if (mag <= 0.0) continue;
            sum = __dadd_rn(sum, pc_term(mag, expo));
        }
    }
    if (t.lead) out[r] = sum;
}

__global__ void k_pc_update(int32_t m, int32_t n, double* rs, double* cs, const double* row_sum,
                            const double* col_sum) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < m && row_sum[t] > 0.0) rs[t] /= safe_sqrt(row_sum[t]);
    if (t < n && col_sum[t] > 0.0) cs[t] /= safe_sqrt(col_sum[t]);
}

// Lanes per row for the elementwise row kernels: the mean row length rounded
// up to a power of two in [1, 32].
inline int row_lanes(int32_t rows, int64_t nnz) {
    const int64_t mean = rows > 0 ? (nnz + rows - 1) / rows : 1;
    int w = 1;
    while (w < 32 && w < mean) w *= 2;
    return w;
}

// Scaled values (v * rs_i) * cs_j (Scaling::apply, scaling.cpp:127-128);
// counts entries the rebuild would drop (|v| <= 1e-14, sparse.cpp:55).
// Elementwise: groups of `lanes` threads walk a row each (four entries per
// lane in flight), so short and long rows both keep the lanes busy.
__global__ void __launch_bounds__(kBlock) k_scale_values(DevCsr M, int transposed, const double* rs,
                                                         const double* cs, double* out,
                                                         unsigned long long* dropped, int lanes) {
    const int64_t tid = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    const int64_t r64 = tid / lanes;
    const int sub = static_cast<int>(tid % lanes);
    unsigned long long d = 0;
    if (r64 < M.rows) {
        const int r = static_cast<int>(r64);
        const int e = M.rp[r + 1];
        const double rr = transposed ? cs[r] : rs[r];
        const double* other = transposed ? rs : cs;
#pragma unroll 4
        for (int k = M.rp[r] + sub; k < e; k += lanes) {
            const double v = transposed ? M.v64[k] * other[M.ci[k]] * rr : M.v64[k] * rr * other[M.ci[k]];
            out[k] = v;
            d += fabs(v) <= 1e-14 ? 1ull : 0ull;
        }
    }
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(dropped, d);
}

// Kept-entry counts per row (the compaction path when entries are dropped).
__global__ void k_kept_counts(DevCsr M, const double* vs, int32_t* cnt) {
    const int r = blockIdx.x * kBlock + threadIdx.x;
    if (r >= M.rows) return;
    int c = 0;
    for (int k = M.rp[r]; k < M.rp[r + 1]; ++k) c += fabs(vs[k]) <= 1e-14 ? 0 : 1;
    cnt[r] = c;
}

__global__ void k_compact(DevCsr M, const double* vs, const int32_t* new_rp, int32_t* ci_out,
                          double* v_out) {
    const int r = blockIdx.x * kBlock + threadIdx.x;
    if (r >= M.rows) return;
    int o = new_rp[r];
    for (int k = M.rp[r]; k < M.rp[r + 1]; ++k) {
        if (fabs(vs[k]) <= 1e-14) continue;
        ci_out[o] = M.ci[k];
        v_out[o] = vs[k];
        ++o;
    }
}

// Scaled problem vectors (scaling.cpp:172-192, then c *= obj_sign, pdhg.cpp:250-252).
__global__ void k_scale_vectors(int32_t m, int32_t n, const double* rs, const double* cs,
                                const double* c, const double* lo, const double* hi,
                                const double* rlo, const double* rhi, double sign, double* c_s,
                                double* lo_s, double* hi_s, double* rlo_s, double* rhi_s) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < n) {
        const double s = cs[t];
        c_s[t] = (c[t] * s) * sign;
        lo_s[t] = fb(lo[t]) ? lo[t] / s : lo[t];
        hi_s[t] = fb(hi[t]) ? hi[t] / s : hi[t];
    }
    if (t < m) {
        const double s = rs[t];
        rlo_s[t] = fb(rlo[t]) ? rlo[t] * s : rlo[t];
        rhi_s[t] = fb(rhi[t]) ? rhi[t] * s : rhi[t];
    }
}

// Norms: [0] |c_s|_2^2, [1] |b_s|_2^2 (b_i = largest finite |scaled row bound|),
// [2] max |c_o|, [3] max finite |row bound|, original. Grid-stride over a capped
// grid, block partials, and a parallel reduction of the partials in the last CTA.
__global__ void __launch_bounds__(kBlock) k_norms(int32_t m, int32_t n, const double* c_s,
                                                  const double* rlo_s, const double* rhi_s,
                                                  const double* c_o, const double* rlo_o,
                                                  const double* rhi_o, double* part,
                                                  IntakeState* is) {
    // sums of squares (q[0], q[1], q[4], q[5]) and maxima (q[2], q[3])
    constexpr int K = kNorms;
    double q[K] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int32_t nmax = m > n ? m : n;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; t < nmax;
         t += static_cast<int64_t>(gridDim.x) * kBlock) {
        if (t < n) {
            q[0] += c_s[t] * c_s[t];
            q[2] = fmax(q[2], fabs(c_o[t]));
            q[4] += c_o[t] * c_o[t];
        }
        if (t < m) {
            double b = 0.0;
            if (fb(rlo_s[t])) b = fabs(rlo_s[t]);
            if (fb(rhi_s[t])) b = smax(b, fabs(rhi_s[t]));
            q[1] += b * b;
            double bo = 0.0;
            if (fb(rlo_o[t])) bo = fabs(rlo_o[t]);
            if (fb(rhi_o[t])) bo = smax(bo, fabs(rhi_o[t]));
            q[3] = fmax(q[3], bo);
            q[5] += bo * bo;
        }
    }
    __shared__ double sh[K][kBlock];
    auto fold = [&]() {
        __syncthreads();
        for (int s = kBlock / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                for (int i = 0; i < K; ++i)
                    sh[i][threadIdx.x] = (i == 2 || i == 3)
                                             ? fmax(sh[i][threadIdx.x], sh[i][threadIdx.x + s])
                                             : sh[i][threadIdx.x] + sh[i][threadIdx.x + s];
            }
            __syncthreads();
        }
    };
    for (int i = 0; i < K; ++i) sh[i][threadIdx.x] = q[i];
    fold();
    if (threadIdx.x == 0)
        for (int i = 0; i < K; ++i) part[K * blockIdx.x + i] = sh[i][0];
    if (!last_cta(&is->ticket)) return;
    // last CTA: each thread folds a strided subset of the partials in block order
    double r[K] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const volatile double* p = part;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock)
        for (int i = 0; i < K; ++i)
            r[i] = (i == 2 || i == 3) ? fmax(r[i], p[K * b + i]) : r[i] + p[K * b + i];
    for (int i = 0; i < K; ++i) sh[i][threadIdx.x] = r[i];
    fold();
    if (threadIdx.x == 0) {
        for (int i = 0; i < K; ++i) is->norms[i] = sh[i][0];
        is->ticket = 0u;
    }
}

}  // namespace

constexpr int kGridCap = 2048;  // grid-stride kernels: enough CTAs to fill every SM

void launch_bin(const int32_t* rp, int32_t rows, int long_threshold, int32_t* long_rows,
                unsigned long long* counters, cudaStream_t s) {
    const int g = nblocks(rows) < kGridCap ? nblocks(rows) : kGridCap;
    if (rows > 0) k_bin<<<g, kBlock, 0, s>>>(rp, rows, long_threshold, long_rows, counters);
}

void launch_uniform_rows(const int32_t* rp, int32_t rows, unsigned* flag, cudaStream_t s) {
    const int g = nblocks(rows) < kGridCap ? nblocks(rows) : kGridCap;
    if (rows > 0) k_uniform_rows<<<g, kBlock, 0, s>>>(rp, rows, flag);
}

void launch_uniform_vec(const double* v, int32_t n, unsigned* flag, cudaStream_t s) {
    const int g = nblocks(n) < kGridCap ? nblocks(n) : kGridCap;
    if (n > 0) k_uniform_vec<<<g, kBlock, 0, s>>>(v, n, flag);
}

void launch_row_extents(const int32_t* rows, int32_t n, const int32_t* rp, int4* out,
                        cudaStream_t s) {
    if (n > 0) k_row_extents<<<nblocks(n), kBlock, 0, s>>>(rows, n, rp, out);
}

void launch_gather_cols(const int32_t* ci, const int64_t* pos, int32_t n, int32_t* out,
                        cudaStream_t s) {
    if (n > 0) k_gather_cols<<<nblocks(n), kBlock, 0, s>>>(ci, pos, n, out);
}

void launch_dense_rows(const int32_t* ci, const int4* ext, int32_t n_ext, int32_t* dense_off,
                       unsigned long long* nnz_dense, cudaStream_t s) {
    if (n_ext > 0)
        k_dense_rows<<<n_ext < 4096 ? n_ext : 4096, kBlock, 0, s>>>(ci, ext, n_ext, dense_off, nnz_dense);
}

void launch_affine_slices(const RowSlices& S, int2* affine, unsigned long long* nnz_affine,
                          cudaStream_t s) {
    if (S.n_slice == 0) return;
    k_affine_slices<<<S.n_slice < 4096 ? S.n_slice : 4096, kBlock, 0, s>>>(S, affine, nnz_affine);
}

void launch_fill_slices(const DevCsr& M, RowSlices S, int32_t* col, float* v32, double* v64,
                        int64_t total, cudaStream_t s) {
    if (S.n_slice == 0 || total == 0) return;
    const int g = S.n_slice < kGridCap ? S.n_slice : kGridCap;
    k_fill_slices<<<g, kBlock, 0, s>>>(M.rp, M.ci, M.v64, M.v32, S, col, v32, v64);
}

void launch_bin_range(const int32_t* rp, int32_t rows, int lo, int hi, int32_t* list,
                      unsigned long long* count, cudaStream_t s) {
    const int g = nblocks(rows) < kGridCap ? nblocks(rows) : kGridCap;
    if (rows > 0) k_bin_range<<<g, kBlock, 0, s>>>(rp, rows, lo, hi, list, count);
}

inline int short_blocks(const DevCsr& M) {
    if (M.n_short == 0) return 0;
    return static_cast<int>((static_cast<int64_t>(M.rows) * M.vw + kBlock - 1) / kBlock);
}

void launch_ruiz_sweep(const DevCsr& A, const DevCsr& AT, double* rs, double* cs,
                       double* row_max, double* col_max, double tol, IntakeState* is,
                       cudaStream_t s) {
    const int sa = short_blocks(A), st = short_blocks(AT);
    if (sa + A.n_long > 0)
        k_ruiz_max<<<sa + A.n_long, kBlock, 0, s>>>(A, 0, rs, cs, is, row_max, sa);
    if (st + AT.n_long > 0)
        k_ruiz_max<<<st + AT.n_long, kBlock, 0, s>>>(AT, 1, rs, cs, is, col_max, st);
    const int32_t nmax = A.rows > AT.rows ? A.rows : AT.rows;
    k_ruiz_update<<<nmax > 0 ? nblocks(nmax) : 1, kBlock, 0, s>>>(A.rows, AT.rows, rs, cs,
                                                                 row_max, col_max, tol, is);
}

void launch_pock_chambolle(const DevCsr& A, const DevCsr& AT, double* rs, double* cs,
                           double* row_sum, double* col_sum, double alpha, cudaStream_t s) {
    // both sums from the factors before this step (scaling.cpp:85-96), then the update
    if (A.rows > 0) k_pc_sum<<<mat_blocks(A), kBlock, 0, s>>>(A, 0, rs, cs, 2.0 - alpha, row_sum);
    if (AT.rows > 0) k_pc_sum<<<mat_blocks(AT), kBlock, 0, s>>>(AT, 1, rs, cs, alpha, col_sum);
    const int32_t nmax = A.rows > AT.rows ? A.rows : AT.rows;
    if (nmax > 0) k_pc_update<<<nblocks(nmax), kBlock, 0, s>>>(A.rows, AT.rows, rs, cs, row_sum, col_sum);
}

void launch_scale_values(const DevCsr& M, int transposed, const double* rs, const double* cs,
                         double* out, unsigned long long* dropped, cudaStream_t s) {
    if (M.rows > 0) {
        const int lanes = row_lanes(M.rows, M.nnz);
        k_scale_values<<<nblocks(static_cast<int64_t>(M.rows) * lanes), kBlock, 0, s>>>(
            M, transposed, rs, cs, out, dropped, lanes);
    }
}

void launch_kept_counts(const DevCsr& M, const double* vs, int32_t* cnt, cudaStream_t s) {
    if (M.rows > 0) k_kept_counts<<<nblocks(M.rows), kBlock, 0, s>>>(M, vs, cnt);
}

void launch_compact(const DevCsr& M, const double* vs, const int32_t* new_rp, int32_t* ci_out,
                    double* v_out, cudaStream_t s) {
    if (M.rows > 0) k_compact<<<nblocks(M.rows), kBlock, 0, s>>>(M, vs, new_rp, ci_out, v_out);
}

void launch_scale_vectors(int32_t m, int32_t n, const double* rs, const double* cs,
                          const double* c, const double* lo, const double* hi, const double* rlo,
                          const double* rhi, double sign, double* c_s, double* lo_s,
                          double* hi_s, double* rlo_s, double* rhi_s, cudaStream_t s) {
    const int32_t nmax = m > n ? m : n;
    if (nmax > 0)
        k_scale_vectors<<<nblocks(nmax), kBlock, 0, s>>>(m, n, rs, cs, c, lo, hi, rlo, rhi, sign,
                                                         c_s, lo_s, hi_s, rlo_s, rhi_s);
}

void launch_validate(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     const double* c, const double* clo, const double* chi, const double* rlo,
                     const double* rhi, int64_t nnz, unsigned* flags, cudaStream_t s) {
    const int lanes = row_lanes(m, nnz);
    const int64_t work = std::max<int64_t>(std::max<int64_t>(m, n), static_cast<int64_t>(m) * lanes);
    int g = work > 0 ? nblocks(work) : 1;
    if (g > kGridCap) g = kGridCap;
    k_validate<<<g, kBlock, 0, s>>>(m, n, rp, ci, v, c, clo, chi, rlo, rhi, lanes, flags);
}

int norms_part_size(int32_t m, int32_t n) { return kNorms * (kGridCap + 1); }

void launch_norms(int32_t m, int32_t n, const double* c_s, const double* rlo_s,
                  const double* rhi_s, const double* c_o, const double* rlo_o,
                  const double* rhi_o, double* part, IntakeState* is, cudaStream_t s) {
    const int32_t nmax = m > n ? m : n;
    int g = nmax > 0 ? nblocks(nmax) : 1;
    if (g > kGridCap) g = kGridCap;
    k_norms<<<g, kBlock, 0, s>>>(m, n, c_s, rlo_s, rhi_s, c_o, rlo_o, rhi_o, part, is);
}

}  // namespace pdhg

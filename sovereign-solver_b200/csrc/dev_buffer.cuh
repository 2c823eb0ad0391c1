// dev_buffer.cuh -- owning device buffers and the resident CSR used by the
// single-LP engine (engine.cu) and the batched engine (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/pdhg_b200.h"
#include "engine.cuh"

namespace pdhg {

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p != nullptr) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count == n && p != nullptr) return cudaSuccess;
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
    }
};

// Owning storage of a RowItems list.
struct ItemsDev {
    DBuf<int4> item;
    DBuf<int2> split;
    DBuf<unsigned int> ticket, fetch;
    DBuf<double> part;
    int32_t n_item = 0;
    RowItems view() const {
        RowItems v;
        v.item = item.p;
        v.split = split.p;
        v.ticket = ticket.p;
        v.part = part.p;
        v.fetch = fetch.p;
        v.n_item = n_item;
        return v;
    }
};

// Owning storage of a LongTiers set.
struct TiersDev {
    DBuf<int32_t> warp_rows0, warp_rows1;
    int32_t n_warp0 = 0, n_warp1 = 0;
    ItemsDev items_long, items_huge, items_warp;
    LongTiers view() const {
        LongTiers t;
        t.warp_rows0 = warp_rows0.p;
        t.warp_rows1 = warp_rows1.p;
        t.n_warp0 = n_warp0;
        t.n_warp1 = n_warp1;
        t.items_long = items_long.view();
        t.items_huge = items_huge.view();
        t.items_warp = items_warp.view();
        return t;
    }
};

// Owning storage of RowSlices.
struct SlicesDev {
    DBuf<int4> slice, item;
    DBuf<int2> split, affine;
    DBuf<int32_t> row, rlen, col;
    DBuf<float> v32;
    DBuf<double> v64, part, cpart;
    DBuf<unsigned int> ticket, fetch, cticket;
    int32_t n_slice = 0, n_item = 0;
    int64_t nnz_affine = 0;  // entries of the affine slices (columns computed)
    RowSlices view() const {
        RowSlices v;
        v.n_slice = n_slice;
        v.n_item = n_item;
        v.slice = slice.p;
        v.row = row.p;
        v.rlen = rlen.p;
        v.col = col.p;
        v.v32 = v32.p;
        v.v64 = v64.p;
        v.item = item.p;
        v.split = split.p;
        v.ticket = ticket.p;
        v.part = part.p;
        v.fetch = fetch.p;
        v.cticket = cticket.p;
        v.cpart = cpart.p;
        v.affine = affine.p;
        return v;
    }
};

struct MatDev {
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;
    DBuf<int32_t> rp, ci, long_rows, wrows, warp_rows0, warp_rows1, dense_off;
    ItemsDev items_long, items_huge, items_warp;
    std::vector<int4> ext;  // host: {row, begin, end, -} of every row above short_max, row order
    SlicesDev slices;
    TiersDev no_slice_tiers;
    DBuf<double> v64;
    DBuf<float> v32;
    DBuf<char> tscratch;  // build_transpose scratch when this matrix is a transpose
    int32_t n_long = 0, n_short = 0, n_wrows = 0, n_mid = 0, n_huge = 0;
    int32_t short_max = kLongRow, n_iter_short = 0, n_warp0 = 0, n_warp1 = 0;
    int vw = 1;
    int32_t rp_stride = 0;  // every row this long (0: not uniform)
    int64_t nnz_dense = 0;  // entries of the dense rows (columns computed)
    DevCsr view() const {
        DevCsr d;
        d.rows = rows;
        d.cols = cols;
        d.nnz = nnz;
        d.rp = rp.p;
        d.ci = ci.p;
        d.v64 = v64.p;
        d.v32 = v32.p;
        d.long_rows = long_rows.p;
        d.n_long = n_long;
        d.n_short = n_short;
        d.vw = vw;
        d.wrows = wrows.p;
        d.n_wrows = n_wrows;
        d.short_max = short_max;
        d.n_iter_short = n_iter_short;
        d.warp_rows0 = warp_rows0.p;
        d.warp_rows1 = warp_rows1.p;
        d.n_warp0 = n_warp0;
        d.n_warp1 = n_warp1;
        d.n_mid = n_mid;
        d.n_huge = n_huge;
        d.items_long = items_long.view();
        d.items_huge = items_huge.view();
        d.items_warp = items_warp.view();
        d.slices = slices.view();
        d.no_slice_tiers = no_slice_tiers.view();
        d.rp_stride = rp_stride;
        d.dense_off = dense_off.p;
        return d;
    }
};

template <class T>
inline cudaError_t upload(DBuf<T>& d, const T* h, size_t n, cudaStream_t s) {
    cudaError_t e = d.alloc(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(d.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s);
}

template <class T>
inline cudaError_t upload(DBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
    return upload(d, h.data(), h.size(), s);
}

template <class T>
inline cudaError_t copy_dev(DBuf<T>& d, const T* src, size_t n, cudaStream_t s) {
    cudaError_t e = d.alloc(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(d.p, src, sizeof(T) * n, cudaMemcpyDeviceToDevice, s);
}

inline cudaError_t to_float(DBuf<float>& d, const DBuf<double>& src, cudaStream_t s) {
    cudaError_t e = d.alloc(src.n);
    if (e != cudaSuccess) return e;
    launch_to_float(src.p, d.p, static_cast<int64_t>(src.n), s);
    return cudaGetLastError();
}

// Opt-in phase timing for load and solve: with PDHG_B200_PHASE_TIMES=1 in the
// environment every mark waits for the stream and prints, to stderr, the host
// wall time since the previous mark. Off (no waits, no output) otherwise.
inline bool phase_times_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("PDHG_B200_PHASE_TIMES");
        return e != nullptr && e[0] == '1';
    }();
    return on;
}

struct PhaseClock {
    bool on;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t;
    explicit PhaseClock(cudaStream_t st)
        : on(phase_times_enabled()), s(st), t(std::chrono::steady_clock::now()) {}
    void mark(const char* what) {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[pdhg phase] %-22s %10.3f ms\n", what,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

inline int cuda_fail(std::string* err, cudaError_t e, const char* what) {
    *err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PDHG_ERR_OUT_OF_MEMORY : PDHG_ERR_BACKEND;
}

// Work items (RowItems) over the rows of `ext` ({row, begin, end, -}, in row
// order) longer than min_len: one item per row of at most seg entries, else
// ceil(len / seg) near-equal segments. seg is min_seg, or more when the rows'
// entries would make more than two items per resident CTA (or warp) of the
// GPU (`resident`): rows are split only as far as filling the GPU needs.
inline int build_items(const std::vector<int4>& ext, int min_len, int min_seg, int resident,
                       ItemsDev& D, cudaStream_t s, std::string* err) {
    int64_t total = 0;
    for (const int4& r : ext)
        if (r.z - r.y > min_len) total += static_cast<int64_t>(r.z) - r.y;
    const int64_t seg = std::max<int64_t>(min_seg, (total + 2 * resident - 1) / (2 * resident));
    std::vector<int4> items;
    std::vector<int2> splits;
    for (const int4& r : ext) {
        const int64_t len = static_cast<int64_t>(r.z) - r.y;
        if (len <= min_len) continue;
        const int64_t nseg = (len + seg - 1) / seg;
        if (nseg <= 1) {
            items.push_back(make_int4(r.x, r.y, r.z, -1));
            continue;
        }
        const int sid = static_cast<int>(splits.size());
        splits.push_back(make_int2(static_cast<int>(items.size()), static_cast<int>(nseg)));
        for (int64_t k = 0; k < nseg; ++k) {
            const int b = r.y + static_cast<int>(len * k / nseg);
            const int e = r.y + static_cast<int>(len * (k + 1) / nseg);
            items.push_back(make_int4(r.x, b, e, sid));
        }
    }
    D.n_item = static_cast<int32_t>(items.size());
    cudaError_t e;
    if ((e = upload(D.item, items.data(), items.size(), s)) != cudaSuccess ||
        (e = upload(D.split, splits.data(), splits.size(), s)) != cudaSuccess ||
        (e = D.ticket.alloc(splits.size())) != cudaSuccess ||
        (e = D.part.alloc(2 * items.size())) != cudaSuccess ||
        (e = D.fetch.alloc(2)) != cudaSuccess)
        return cuda_fail(err, e, "build_items");
    if (!splits.empty()) cudaMemsetAsync(D.ticket.p, 0, sizeof(unsigned int) * splits.size(), s);
    cudaMemsetAsync(D.fetch.p, 0, 2 * sizeof(unsigned int), s);
    // the host vectors are read by the copies above before they go out of scope
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "build_items");
    return PDHG_OK;
}

// Row binning on the device: long-row list, short-row count, lanes per short
// row (about half the mean short-row length, a power of two in [1, 32]), the
// warp-row list of the ordered kernels, and the throughput kernels' tiers:
// short rows up to short_max, the two warp-row lists and the CTA work items.
inline int bin_matrix(MatDev& M, cudaStream_t s, std::string* err) {
    cudaError_t e = M.long_rows.alloc(static_cast<size_t>(M.rows) + 1);
    if (e != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    if ((e = M.wrows.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.warp_rows0.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.warp_rows1.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess)
        return cuda_fail(err, e, "bin_matrix");
    DBuf<unsigned long long> cnt;
    if ((e = cnt.alloc(9)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    cudaMemsetAsync(cnt.p, 0, 9 * sizeof(unsigned long long), s);
    launch_bin(M.rp.p, M.rows, kLongRow, M.long_rows.p, cnt.p, s);
    launch_bin(M.rp.p, M.rows, kWarpRow, M.wrows.p, cnt.p + 3, s);
    // rows all of one length: the short-row kernel computes their extents
    launch_uniform_rows(M.rp.p, M.rows, reinterpret_cast<unsigned*>(cnt.p + 8), s);
    int32_t rp01[2] = {0, 0};
    if (M.rows > 0) cudaMemcpyAsync(rp01, M.rp.p, sizeof rp01, cudaMemcpyDeviceToHost, s);
    unsigned long long h[9];
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_long = static_cast<int32_t>(h[0]);
    M.n_short = static_cast<int32_t>(h[1]);
    M.n_wrows = static_cast<int32_t>(h[3]);
    M.rp_stride = (M.rows > 0 && h[8] == 0 && rp01[0] == 0) ? rp01[1] : 0;
    const double mean = h[1] > 0 ? static_cast<double>(h[2]) / static_cast<double>(h[1]) : 0.0;
    int w = 1;
    while (w < 32 && 2.0 * w <= mean / 2.0 + 1e-9) w *= 2;
    M.vw = w;
    // lane groups take rows of up to 16 lanes' worth (a few unrolled rounds
    // per lane); longer rows go to a warp each
    M.short_max = std::min(kLongRow, std::max(kWarpRow, 16 * w));
    launch_bin_range(M.rp.p, M.rows, M.short_max, kLongRow, M.warp_rows0.p, cnt.p + 6, s);
    launch_bin_range(M.rp.p, M.rows, M.short_max, kHugeRow, M.warp_rows1.p, cnt.p + 7, s);
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_warp0 = static_cast<int32_t>(h[6]);
    M.n_warp1 = static_cast<int32_t>(h[7]);

    // extents of every row above short_max (warp_rows0 + long rows), in row
    // order (the binning kernels append in arrival order)
    std::vector<int4> ext(static_cast<size_t>(M.n_long) + static_cast<size_t>(M.n_warp0));
    if (!ext.empty()) {
        DBuf<int4> d_ext;
        if ((e = d_ext.alloc(ext.size())) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
        launch_row_extents(M.long_rows.p, M.n_long, M.rp.p, d_ext.p, s);
        launch_row_extents(M.warp_rows0.p, M.n_warp0, M.rp.p, d_ext.p + M.n_long, s);
        cudaMemcpyAsync(ext.data(), d_ext.p, sizeof(int4) * ext.size(), cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
        std::sort(ext.begin(), ext.end(), [](const int4& a, const int4& b) { return a.x < b.x; });
    }
    M.ext = ext;
    M.slices.n_slice = 0;
    M.slices.n_item = 0;
    M.n_huge = 0;
    for (const int4& r : ext) M.n_huge += (r.z - r.y > kHugeRow) ? 1 : 0;
    M.n_mid = M.n_long - M.n_huge;
    M.n_iter_short = M.rows - M.n_warp1 - M.n_huge;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms = std::max(sms, 1);
    const int resident = 4 * sms;  // the long-row kernel's CTAs per SM
    int rc = build_items(ext, kLongRow, kSegLen, resident, M.items_long, s, err);
    if (rc != PDHG_OK) return rc;
    rc = build_items(ext, kHugeRow, kSegLen, resident, M.items_huge, s, err);
    if (rc != PDHG_OK) return rc;
    return build_items(ext, M.short_max, kWarpSegLen, 32 * sms, M.items_warp, s, err);
}

// The long-row tiers over the rows of `ext` (row order, all above short_max),
// built on the host: warp-row lists and the three item lists.
inline int build_tiers(const std::vector<int4>& ext, int short_max, int sms, TiersDev& T,
                       cudaStream_t s, std::string* err) {
    std::vector<int32_t> w0, w1;
    for (const int4& r : ext) {
        const int len = r.z - r.y;
        if (len > short_max && len <= kLongRow) w0.push_back(r.x);
        if (len > short_max && len <= kHugeRow) w1.push_back(r.x);
    }
    T.n_warp0 = static_cast<int32_t>(w0.size());
    T.n_warp1 = static_cast<int32_t>(w1.size());
    cudaError_t e;
    if ((e = upload(T.warp_rows0, w0, s)) != cudaSuccess ||
        (e = upload(T.warp_rows1, w1, s)) != cudaSuccess)
        return cuda_fail(err, e, "build_tiers");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "build_tiers");
    int rc = build_items(ext, kLongRow, kSegLen, 4 * sms, T.items_long, s, err);
    if (rc != PDHG_OK) return rc;
    rc = build_items(ext, kHugeRow, kSegLen, 4 * sms, T.items_huge, s, err);
    if (rc != PDHG_OK) return rc;
    return build_items(ext, short_max, kWarpSegLen, 32 * sms, T.items_warp, s, err);
}

// Distinct 128-byte lines (32 four-byte entries) among 32 column indices.
inline int lines_of(const int32_t* c) {
    int32_t l[32];
    for (int i = 0; i < 32; ++i) l[i] = c[i] >> 5;
    std::sort(l, l + 32);
    return static_cast<int>(std::unique(l, l + 32) - l);
}

constexpr int kSliceMinLen = 256;  // rows shorter than this are not worth a slice

// Row slices of a scaled matrix (after bin_matrix, values in v64 and v32).
// Candidates: runs of 32 consecutive rows of M.ext whose lengths are within
// 5% of each other and at least kSliceMinLen. For each, column indices are
// sampled at four positions k: across the 32 rows at k (slice order) and
// along the first row from k (row order); a candidate becomes a slice when a
// 32-wide gather in slice order touches at most a quarter of the 128-byte
// lines it touches in row order. Then the lane-interleaved copy, the warp
// items (k-chunks, split like rows when a slice needs several) and the long-
// row tiers of the remaining rows.
inline int build_slices(MatDev& M, cudaStream_t s, std::string* err) {
    SlicesDev& S = M.slices;
    S.n_slice = 0;
    S.nnz_affine = 0;
    S.n_item = 0;
    const std::vector<int4>& ext = M.ext;
    std::vector<size_t> cand;
    std::vector<int> cand_lo;
    for (size_t i = 0; i + 32 <= ext.size();) {
        int lo = 0x7fffffff, hi = 0;
        for (size_t j = i; j < i + 32; ++j) {
            const int len = ext[j].z - ext[j].y;
            lo = std::min(lo, len);
            hi = std::max(hi, len);
        }
        if (lo >= kSliceMinLen && static_cast<int64_t>(lo) * 20 >= static_cast<int64_t>(hi) * 19) {
            cand.push_back(i);
            cand_lo.push_back(lo);
            i += 32;
        } else {
            ++i;
        }
    }
    if (cand.empty()) return PDHG_OK;
    // sampled positions: per candidate, 4 x (32 across rows + 32 along row 0)
    constexpr int kSamples = 4;
    std::vector<int64_t> pos;
    pos.reserve(cand.size() * kSamples * 64);
    for (size_t c = 0; c < cand.size(); ++c) {
        const int lo = cand_lo[c];
        for (int q = 0; q < kSamples; ++q) {
            const int k = static_cast<int>(static_cast<int64_t>(lo - 32) * q / (kSamples - 1));
            for (int l = 0; l < 32; ++l) pos.push_back(static_cast<int64_t>(ext[cand[c] + l].y) + k);
            for (int l = 0; l < 32; ++l) pos.push_back(static_cast<int64_t>(ext[cand[c]].y) + k + l);
        }
    }
    std::vector<int32_t> cols(pos.size());
    {
        DBuf<int64_t> d_pos;
        DBuf<int32_t> d_cols;
        cudaError_t e;
        if ((e = upload(d_pos, pos, s)) != cudaSuccess || (e = d_cols.alloc(pos.size())) != cudaSuccess)
            return cuda_fail(err, e, "build_slices");
        launch_gather_cols(M.ci.p, d_pos.p, static_cast<int32_t>(pos.size()), d_cols.p, s);
        cudaMemcpyAsync(cols.data(), d_cols.p, sizeof(int32_t) * cols.size(), cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "build_slices");
    }
    std::vector<size_t> chosen;
    for (size_t c = 0; c < cand.size(); ++c) {
        int across = 0, along = 0;
        for (int q = 0; q < kSamples; ++q) {
            const int32_t* b = cols.data() + (c * kSamples + q) * 64;
            across += lines_of(b);
            along += lines_of(b + 32);
        }
        if (4 * across <= along) chosen.push_back(cand[c]);
    }
    if (chosen.empty()) return PDHG_OK;

    // slice metadata and the lane-interleaved copy
    const int ns = static_cast<int>(chosen.size());
    std::vector<int4> meta(static_cast<size_t>(ns));
    std::vector<int32_t> row(32 * static_cast<size_t>(ns)), rlen(32 * static_cast<size_t>(ns));
    int64_t total = 0, ksteps = 0;
    for (int sl = 0; sl < ns; ++sl) {
        int len = 0;
        for (int l = 0; l < 32; ++l) {
            const int4& r = ext[chosen[static_cast<size_t>(sl)] + static_cast<size_t>(l)];
            row[32 * static_cast<size_t>(sl) + l] = r.x;
            rlen[32 * static_cast<size_t>(sl) + l] = r.z - r.y;
            len = std::max(len, r.z - r.y);
        }
        if (total + 32 * static_cast<int64_t>(len) > 0x7fffffffLL) break;  // int offsets
        meta[static_cast<size_t>(sl)] = make_int4(len, static_cast<int>(total), 32, 0);
        total += 32 * static_cast<int64_t>(len);
        ksteps += len;
        S.n_slice = sl + 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms = std::max(sms, 1);
    // warp items: k-chunks of at least 32 steps, about four per resident warp
    // (the slice kernel is persistent and claims items one by one)
    const int64_t resident = 32LL * sms;
    int64_t chunk = std::max<int64_t>(32, (ksteps + 4 * resident - 1) / (4 * resident));
    chunk = (chunk + 7) / 8 * 8;
    std::vector<int4> items;
    std::vector<int2> splits;
    for (int sl = 0; sl < S.n_slice; ++sl) {
        const int len = meta[static_cast<size_t>(sl)].x;
        const int nchunk = static_cast<int>((len + chunk - 1) / chunk);
        if (nchunk <= 1) {
            items.push_back(make_int4(sl, 0, len, -1));
            continue;
        }
        const int sid = static_cast<int>(splits.size());
        splits.push_back(make_int2(static_cast<int>(items.size()), nchunk));
        for (int q = 0; q < nchunk; ++q)
            items.push_back(make_int4(sl, static_cast<int>(q * chunk),
                                      static_cast<int>(std::min<int64_t>(len, (q + 1) * chunk)), sid));
    }
    S.n_item = static_cast<int32_t>(items.size());
    cudaError_t e;
    meta.resize(static_cast<size_t>(S.n_slice));
    row.resize(32 * static_cast<size_t>(S.n_slice));
    rlen.resize(32 * static_cast<size_t>(S.n_slice));
    if ((e = upload(S.slice, meta, s)) != cudaSuccess || (e = upload(S.row, row, s)) != cudaSuccess ||
        (e = upload(S.rlen, rlen, s)) != cudaSuccess || (e = S.col.alloc(static_cast<size_t>(total))) != cudaSuccess ||
        (e = S.v32.alloc(static_cast<size_t>(total))) != cudaSuccess ||
        (e = S.v64.alloc(static_cast<size_t>(total))) != cudaSuccess ||
        (e = upload(S.item, items, s)) != cudaSuccess || (e = upload(S.split, splits, s)) != cudaSuccess ||
        (e = S.ticket.alloc(splits.size())) != cudaSuccess ||
        (e = S.part.alloc(32 * items.size())) != cudaSuccess ||
        (e = S.cticket.alloc(splits.size())) != cudaSuccess ||
        (e = S.cpart.alloc(64 * items.size())) != cudaSuccess ||
        (e = S.fetch.alloc(2)) != cudaSuccess)
        return cuda_fail(err, e, "build_slices");
    if (!splits.empty()) {
        cudaMemsetAsync(S.ticket.p, 0, sizeof(unsigned int) * splits.size(), s);
        cudaMemsetAsync(S.cticket.p, 0, sizeof(unsigned int) * splits.size(), s);
    }
    cudaMemsetAsync(S.fetch.p, 0, 2 * sizeof(unsigned int), s);
    launch_fill_slices(M.view(), S.view(), S.col.p, S.v32.p, S.v64.p, total, s);
    {
        DBuf<unsigned long long> cnt;
        unsigned long long h = 0;
        if ((e = S.affine.alloc(static_cast<size_t>(S.n_slice))) != cudaSuccess ||
            (e = cnt.alloc(1)) != cudaSuccess ||
            (e = cudaMemsetAsync(cnt.p, 0, sizeof h, s)) != cudaSuccess)
            return cuda_fail(err, e, "build_slices");
        launch_affine_slices(S.view(), S.affine.p, cnt.p, s);
        if ((e = cudaMemcpyAsync(&h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(err, e, "build_slices");
        S.nnz_affine = static_cast<int64_t>(h);
    }

    // the long-row tiers without the rows of the slices kept
    std::vector<char> in_slice(ext.size(), 0);
    for (int sl = 0; sl < S.n_slice; ++sl)
        for (size_t l = 0; l < 32; ++l) in_slice[chosen[static_cast<size_t>(sl)] + l] = 1;
    std::vector<int4> rest;
    rest.reserve(ext.size());
    for (size_t i = 0; i < ext.size(); ++i)
        if (!in_slice[i]) rest.push_back(ext[i]);
    return build_tiers(rest, M.short_max, sms, M.no_slice_tiers, s, err);
}

// Dense rows among the rows above short_max (k_dense_rows); none listed, no
// array.
inline int build_dense_rows(MatDev& M, cudaStream_t s, std::string* err) {
    const char* knob = std::getenv("PDHG_B200_DENSE_ROWS");  // "0": load every column index
    M.nnz_dense = 0;
    if (M.ext.empty() || (knob != nullptr && knob[0] == '0')) {
        M.dense_off.release();
        return PDHG_OK;
    }
    DBuf<int4> d_ext;
    DBuf<unsigned long long> cnt;
    unsigned long long h = 0;
    cudaError_t e;
    if ((e = upload(d_ext, M.ext, s)) != cudaSuccess ||
        (e = M.dense_off.alloc(static_cast<size_t>(M.rows))) != cudaSuccess ||
        (e = cudaMemsetAsync(M.dense_off.p, 0x80, sizeof(int32_t) * static_cast<size_t>(M.rows), s)) !=
            cudaSuccess ||
        (e = cnt.alloc(1)) != cudaSuccess || (e = cudaMemsetAsync(cnt.p, 0, sizeof h, s)) != cudaSuccess)
        return cuda_fail(err, e, "build_dense_rows");
    launch_dense_rows(M.ci.p, d_ext.p, static_cast<int32_t>(M.ext.size()), M.dense_off.p, cnt.p, s);
    if ((e = cudaMemcpyAsync(&h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(err, e, "build_dense_rows");
    M.nnz_dense = static_cast<int64_t>(h);
    return PDHG_OK;
}

// row_ptr structure on the host (rows + 1 reads): starts at 0, ends at nnz,
// non-decreasing. Every device kernel that walks rows relies on it.
inline bool row_ptr_ok(int32_t rows, int64_t nnz, const int32_t* rp) {
    if (rp[0] != 0 || rp[rows] != nnz) return false;
    for (int32_t r = 0; r < rows; ++r)
        if (rp[r] > rp[r + 1]) return false;
    return true;
}

// A's arrays to the device, read in place from the caller's host buffers.
inline int upload_csr(int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp,
                      const int32_t* ci, const double* v, MatDev& M, cudaStream_t s,
                      std::string* err) {
    cudaError_t e;
    M.rows = rows;
    M.cols = cols;
    M.nnz = nnz;
    if ((e = upload(M.rp, rp, static_cast<size_t>(rows) + 1, s)) != cudaSuccess ||
        (e = upload(M.ci, ci, static_cast<size_t>(nnz), s)) != cudaSuccess ||
        (e = upload(M.v64, v, static_cast<size_t>(nnz), s)) != cudaSuccess)
        return cuda_fail(err, e, "upload_csr");
    return PDHG_OK;
}

// The device problem checks (launch_validate) on data already resident;
// *flags gets the OR of the failing kinds (0: nothing failed).
inline int device_checks(const MatDev& M, const double* c, const double* clo, const double* chi,
                         const double* rlo, const double* rhi, unsigned* flags, cudaStream_t s,
                         std::string* err) {
    DBuf<unsigned> f;
    cudaError_t e = f.alloc(1);
    if (e != cudaSuccess) return cuda_fail(err, e, "device_checks");
    cudaMemsetAsync(f.p, 0, sizeof(unsigned), s);
    launch_validate(M.rows, M.cols, M.rp.p, M.ci.p, M.v64.p, c, clo, chi, rlo, rhi, M.nnz, f.p, s);
    cudaMemcpyAsync(flags, f.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "device_checks");
    return PDHG_OK;
}

// A^T built on the device from the resident A, then both binned.
inline int finish_matrix(MatDev& M, MatDev& MT, cudaStream_t s, std::string* err) {
    cudaError_t e;
    PhaseClock pc(s);
    MT.rows = M.cols;
    MT.cols = M.rows;
    MT.nnz = M.nnz;
    if ((e = MT.rp.alloc(static_cast<size_t>(M.cols) + 1)) != cudaSuccess ||
        (e = MT.ci.alloc(static_cast<size_t>(M.nnz))) != cudaSuccess ||
        (e = MT.v64.alloc(static_cast<size_t>(M.nnz))) != cudaSuccess)
        return cuda_fail(err, e, "finish_matrix");
    if ((e = MT.tscratch.alloc(transpose_scratch_bytes(M.rows, M.cols, M.nnz))) != cudaSuccess)
        return cuda_fail(err, e, "finish_matrix");
    TransposeOut out{MT.rp.p, MT.ci.p, MT.v64.p};
    if (build_transpose(M.rows, M.cols, M.nnz, M.rp.p, M.ci.p, M.v64.p, out, MT.tscratch.p, s) != 0)
        return cuda_fail(err, cudaGetLastError(), "build_transpose");
    pc.mark("matrix: transpose");
    int rc = bin_matrix(M, s, err);
    if (rc != PDHG_OK) return rc;
    rc = bin_matrix(MT, s, err);
    pc.mark("matrix: bins");
    return rc;
}

// A matrix on its own (no problem around it): row_ptr checked on the host and
// the column indices on the device, then A^T and the bins. A matrix whose
// structure would send a kernel out of bounds returns PDHG_ERR_INVALID_ARGUMENT
// before any kernel indexes by it; unsorted columns and non-finite values are
// the caller's (the product is formed as given).
inline int upload_matrix(int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp,
                         const int32_t* ci, const double* v, MatDev& M, MatDev& MT,
                         cudaStream_t s, std::string* err) {
    if (!row_ptr_ok(rows, nnz, rp)) {
        *err = "invalid CSR matrix: row_ptr must start at 0, end at nnz and not decrease";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    int rc = upload_csr(rows, cols, nnz, rp, ci, v, M, s, err);
    if (rc != PDHG_OK) return rc;
    unsigned flags = 0;
    rc = device_checks(M, nullptr, nullptr, nullptr, nullptr, nullptr, &flags, s, err);
    if (rc != PDHG_OK) return rc;
    if (flags & 4u) {
        *err = "invalid CSR matrix: column index out of range";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    return finish_matrix(M, MT, s, err);
}

}  // namespace pdhg

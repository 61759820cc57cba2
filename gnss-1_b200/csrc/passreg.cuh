// passreg.cuh -- strided x / y passes with register-resident column
// transforms (N = 64, 96, 128, 192, 256, 512).
//
// Same contract as k_pass (PassSpec / PassPtrs: tiles of NB columns x N rows,
// kept / compact rows and outer indices, up to two outputs per tile, each the
// transform of the tile times a spectral multiplier, optional dealias mask),
// with a different schedule: warp w owns column w of the tile and transforms
// it in registers with zr_fft (one transpose, inside the warp's column of the
// output tile), so a column crosses shared memory three times (load,
// transpose, store) and the block synchronises per tile and per output
// instead of per radix stage.
//   tile rows are padded to NB + 1 elements: a warp reading one column and a
//   half-warp pair writing one row are both free of bank conflicts;
//   the next tile is copied with cp.async (rows the spec does not keep are
//   neither copied nor read) while the current one is transformed;
//   the dealias mask keeps rows whose |index| is at most a bound computed
//   once per tile and column (k^2 grows with |k_row|), with the reference's
//   test k^2 > kmax^2 (solver.cu:36) evaluated in the reference's order;
//   results go through the output tile to coalesced row stores; a second
//   output of the same tile reloads the input column from shared memory;
//   per-element bookkeeping is kept out of the element loops (a per-lane
//   mask of the rows it loads, the multiplier chosen once per output,
//   32-bit store offsets).
#pragma once
#include "zreg.cuh"

namespace gnss {

template <typename T, int N> struct PRCfg {
    using Z = ZRCfg<T, N>;
    static constexpr int NB = PassCfg<T, N>::NB;          // columns per tile (as k_pass) = warps per block
    static constexpr int NT = NB * 32;
    static constexpr int LD = NB + 1;                     // padded row
    static constexpr int TILE = N * LD;
    // two input tiles (the copy pipeline) and one output tile
    static constexpr int TWR = Z::rows(true);            // twiddle rows (the full step-A table in FP32)
    static constexpr int SMEM = (3 * TILE + TWR * 32) * (int)sizeof(V2<T>);
};

// zr_fft's transpose inside the warp's own column of the output tile: row k1
// of the transpose is rows 32 k1 .. 32 k1 + 31 of the column, entry i at
// i ^ (2 k1) for G = 2 and i ^ (4 k1) for G = 4 (XOR swizzle: with the odd
// row pitch LD, both the stores and the transposed loads of a warp are free
// of bank conflicts).
template <typename T, int N> struct ColScratch {
    __device__ __forceinline__ int operator()(int k1, int i) const {
        constexpr int G = ZRCfg<T, N>::G;
        return (32 * k1 + (i ^ ((G * k1) & 31))) * PRCfg<T, N>::LD;
    }
};

// Row of the output tile that holds transform row r.  With lane shuffles a
// lane ends holding rows q + E j (j = bitrev5(lane)); storing row q + E j at
// tile row 32 q + j makes a warp's stores of one q land in distinct bank
// pairs (row r itself would put 32 / E lanes on each, with the pitch LD).
// With the transpose, a warp's stores of one q put lane group j = lane % G on
// rows E^2 sigma(j) apart (zr_out_index), all on the same banks; rotating
// block b = r / E^2 of the rows by b RS rows puts the groups that share a
// wavefront (8 lanes of 16 bytes, 16 of 8) on distinct banks (2x fewer
// wavefronts for N = 512, 4x for N = 256).  Measured at 512^3 (FP64, two
// scalars): passes 8.39 -> 8.04 ms per step; at 256^3 FP64 1.39 -> 1.17 ms,
// FP32 0.756 -> 0.714 ms.  FP32 with N = 512 keeps row r: its conflicts are
// 2-way and its passes issue-bound, and the rotation made them 4% slower.
template <typename T, int N> __device__ __forceinline__ int pr_tile_row(int r) {
    using Z = ZRCfg<T, N>;
    if constexpr (Z::SHFL) {
        return (r % Z::E) * 32 + r / Z::E;
    } else if constexpr (sizeof(T) == 4 && Z::E == 16) {
        return r;
    } else {
        constexpr int B = Z::E * Z::E, RS = Z::E / (sizeof(T) == 8 ? 4 : 2);
        const int b = r / B;
        return b * B + (r % B + b * RS) % B;
    }
}

// |row index| of a transform row (the Nyquist row counts as N/2)
template <int N> __device__ __forceinline__ int row_dist(int r) { return r <= N / 2 ? r : N - r; }

template <typename T, int N, int SIGN, bool MB = false>
__global__ void __launch_bounds__(PRCfg<T, N>::NT, (N <= 192 && sizeof(T) == 4) ? 2 : 1)
k_passr(const __grid_constant__ PassPtrs<T> P, const __grid_constant__ PassSpec sp, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    using C = PRCfg<T, N>;
    using Z = ZRCfg<T, N>;
    constexpr int NB = C::NB, NT = C::NT, LD = C::LD, TILE = C::TILE, E = Z::E;
    constexpr int RSTEP = NT / NB;   // rows per copy sweep (32)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tiles = reinterpret_cast<V *>(smem_raw);
    V *outt = tiles + 2 * TILE;
    V *tws = outt + TILE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = sp.outer.count() * sp.ncolblk;
    const int mitems = sp.nin * ntiles;   // items of one member
    const long long nitems = MB ? (long long)sp.nmem * mitems : (long long)mitems;
    long long item = blockIdx.x;
    if (item >= nitems) return;
    for (int i = tid; i < C::TWR * 32; i += NT) tws[i] = tw[Z::tw_index(i, true)];
    // work items fit in 32 bits (members x inputs x outer indices x column blocks), so they are decoded with
    // 32-bit divisions
    auto decode = [&](long long it, int &mi, int &fi, int &oc, int &o, int &c0) {
        const int i32 = (int)it;
        mi = MB ? i32 / mitems : 0;   // member of a batch (MB)
        const int r = MB ? i32 - mi * mitems : i32;
        fi = r / ntiles;
        const int t = r - fi * ntiles;
        oc = t / sp.ncolblk;
        o = sp.outer.expand(oc);
        c0 = (t - oc * sp.ncolblk) * NB;
    };
    // copy of one tile: thread -> column tid % NB, rows tid / NB + 32 k (kept rows only).  The rows a thread
    // copies, their source offsets within a tile (32-bit: a tile spans < 2^31 elements) and which are kept are
    // the same for every tile of the launch.
    static_assert(N / RSTEP <= 32, "one kept-row bit per copy sweep");
    unsigned prow = 0;   // bit k: row tid / NB + RSTEP k is kept
    for (int k = 0; k < N / RSTEP; ++k) prow |= (sp.row_in.kept(tid / NB + RSTEP * k) ? 1u : 0u) << k;
    const int s_row = (int)sp.s_row;
    auto prefetch = [&](long long it, V *dst) {
        int mi, fi, oc, o, c0;
        decode(it, mi, fi, oc, o, c0);
        const V *src = P.in[fi] + (MB ? mi * sp.ms_in : 0LL) + (long long)(sp.outer_in_compact ? oc : o) * sp.s_out + c0;
        const int b = tid % NB;
        if (c0 + b >= sp.ncols) return;
#pragma unroll 4
        for (int k = 0; k < N / RSTEP; ++k) {
            if (!((prow >> k) & 1u)) continue;
            const int row = tid / NB + RSTEP * k;
            const int r = sp.row_in_compact ? sp.row_in.compact(row) : row;
            const V *p = src + r * s_row + b;
            if constexpr (sizeof(T) == 8) cp_async16(dst + row * LD + b, p, 16);
            else cp_async8(dst + row * LD + b, p, 8);
        }
    };
    pdl_wait();
    prefetch(item, tiles);
    cp_async_commit();
    int buf = 0;
    const int b = warp;   // this warp's column
    V *col = outt + b;    // this warp's column of the output tile (also its transpose space)
    // rows lane + 32 m this lane loads: bit m set when the spec keeps the row (fixed for the launch)
    unsigned keptm = 0;
#pragma unroll
    for (int m = 0; m < E; ++m) keptm |= (sp.row_in.kept(lane + 32 * m) ? 1u : 0u) << m;
    for (; item < nitems; item += gridDim.x) {
        cp_async_wait<0>();
        __syncthreads();   // current tile landed; the other input tile and the output tile are free
        const long long next = item + gridDim.x;
        if (next < nitems) prefetch(next, tiles + (buf ^ 1) * TILE);
        cp_async_commit();
        int mi, fi, oc, o, c0;
        decode(item, mi, fi, oc, o, c0);
        const V *cur = tiles + buf * TILE;
        const bool col_ok = c0 + b < sp.ncols;
        const double k_out = sp.n_out ? wavenum(o, sp.n_out, sp.dk_out) : 0.0;
        const double kc = wavenum(c0 + b, sp.n_col, sp.dk_col);
        // rows kept by the dealias mask: |row index| <= dmax (prefix by monotonicity of k^2)
        unsigned okm = col_ok ? keptm : 0u;
        if (sp.mask) {
            int cnt = 0;
            for (int d0 = 0; d0 <= N / 2; d0 += 32) {
                const int d = d0 + lane;
                const bool ok = d <= N / 2 && !(ksq3(sp.dk_row * (double)d, k_out, kc) > sp.kmax2);
                cnt += __popc(__ballot_sync(0xffffffffu, ok));
            }
            const int dmax = cnt - 1;
#pragma unroll
            for (int m = 0; m < E; ++m)
                if (row_dist<N>(lane + 32 * m) > dmax) okm &= ~(1u << m);
        }
        const long long dbase = (MB ? mi * sp.ms_out : 0LL) + (long long)(sp.outer_out_compact ? oc : o) * sp.d_out + c0;
        const int out_cols = sp.out_ncols - c0;
        const int nv = sp.nvar[fi];
        for (int v = 0; v < nv; ++v) {
            const int mul = sp.vmul[fi][v];
            V x[E];
#pragma unroll
            for (int m = 0; m < E; ++m) x[m] = ((okm >> m) & 1u) ? cur[(lane + 32 * m) * LD + b] : V{T(0), T(0)};
            if (mul == V_IK_ROW) {
#pragma unroll
                for (int m = 0; m < E; ++m) {
                    const int ir = lane + 32 * m;   // row index; its wavenumber (Nyquist negative)
                    const T kr = sizeof(T) == 8 ? (T)wavenum(ir, sp.n_row, sp.dk_row)
                                                : (T)sp.dk_row * (T)(ir < sp.n_row / 2 ? ir : ir - sp.n_row);
                    x[m] = V{-kr * x[m].y, kr * x[m].x};
                }
            } else if (mul == V_IK_OUT || mul == V_IK_COL) {
                const T kk = (T)(mul == V_IK_OUT ? k_out : kc);
#pragma unroll
                for (int m = 0; m < E; ++m) x[m] = V{-kk * x[m].y, kk * x[m].x};
            } else if (mul == V_LAP) {
#pragma unroll
                for (int m = 0; m < E; ++m) {
                    const T k2 = (T)ksq3(wavenum(lane + 32 * m, sp.n_row, sp.dk_row), k_out, kc);
                    x[m] = V{-k2 * x[m].x, -k2 * x[m].y};
                }
            }
            zr_fft<T, N, SIGN, ColScratch<T, N>, true>(lane, x, col, tws, ColScratch<T, N>{});
            if constexpr (Z::SHFL) {
                const int j = (int)(__brev((unsigned)lane) >> 27);
#pragma unroll
                for (int q = 0; q < E; ++q) col[(32 * q + j) * LD] = x[q];   // pr_tile_row(q + E j)
            } else {
#pragma unroll
                for (int q = 0; q < E; ++q) col[pr_tile_row<T, N>(zr_out_index<T, N>(lane, q)) * LD] = x[q];
            }
            __syncthreads();   // output tile complete
            V *dst = P.out[sp.vout[fi][v]] + dbase + tid % NB;
            if (tid % NB < out_cols) {
                const int nrow = sp.row_out.count();
                const int drow = (int)sp.d_row;   // row pitch of the destination (< 2^31 elements per tile)
                const V *src = outt + tid % NB;
                for (int rc = tid / NB; rc < nrow; rc += RSTEP) {
                    const int row = sp.row_out.expand(rc);
                    const int r = sp.row_out_compact ? rc : row;
                    dst[r * drow] = src[pr_tile_row<T, N>(row) * LD];
                }
            }
            if (v + 1 < nv) __syncthreads();   // output tile free for the next output
        }
        buf ^= 1;
    }
    cp_async_wait<0>();
}

}  // namespace gnss

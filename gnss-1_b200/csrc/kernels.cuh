// kernels.cuh -- the B200 kernels of the pseudospectral step.
//
//   k_pass      x / y axis C2C pass over [outer][row][col] tiles, persistent
//               and software-pipelined (cp.async double buffering); every
//               input tile is read once and may yield two outputs with
//               different spectral multipliers (derivatives), optionally
//               dealiased, optionally transposed on store.
//   k_zpass     z axis R2C / C2R over pairs of contiguous lines (a + ib).
//   k_zphys     fused z C2R of all physical quantities of a line pair, the
//               nonlinear products (omega x u, u.grad s, colloid term) and the
//               z R2C of the products -- the physical fields never touch HBM.
//   k_update    fused spectral sweep: projection, scalar sign, k=0 rule,
//               dealias mask and the CN/AB2 or IF-RK3 update with history.
//   k_stats_*   deterministic compensated statistics reductions.
//   elementwise kernels mirroring the reference's individual operators.
#pragma once
#include "async.cuh"
#include "fft.cuh"

namespace gnss {

constexpr int MAXF = 16;

template <typename T> struct FieldSet { V2<T> *p[MAXF]; };

struct Geom {
    int nx, ny, nz, nz2;
    double dkx, dky, dkz;   // 2 pi / L per axis
    double kmax2;           // (alias_filter * nx * pi / lx)^2
};

// initialize.cu:678-691: k_i = (2 pi / L) * i for i < n/2, else (2 pi / L) * (i - n)
__device__ __forceinline__ double wavenum(int i, int n, double dk) {
    return (i < n / 2) ? dk * (double)i : dk * ((double)i - (double)n);
}
// k_sq in the reference's evaluation order (solver.cu:27)
__device__ __forceinline__ double ksq3(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// ------------------------------------------------------------ strided pass
// A pass transforms along one axis of a field viewed as [outer][row][col]
// (row = the transform index, col = the contiguous kz index).  Work items are
// (input field, tile) with a tile of NB columns x N rows, rows of 128 bytes.
// Every input tile is read from HBM once and may produce up to two outputs,
// each the transform of the tile times a spectral multiplier:
//   V_ONE 1, V_IK_ROW i k_row, V_IK_OUT i k_outer, V_IK_COL i k_col,
//   V_LAP -(k_row^2 + k_outer^2 + k_col^2),
// optionally after the dealias mask k^2 > kmax^2 -> 0 (all three wavenumbers
// are known in the first, spectral-side pass).  Outputs are written with
// their own strides (a transposed store for the x passes).
enum : signed char { V_ONE = 0, V_IK_ROW = 1, V_IK_OUT = 2, V_IK_COL = 3, V_LAP = 4 };

// Kept indices of one axis under the spherical truncation: {0..K} and
// {n-K..n-1}; K < 0 keeps every index.  Compact storage numbers the kept
// indices 0..2K in order.
struct KeepMap {
    int n, K;
    __host__ __device__ __forceinline__ bool kept(int i) const { return K < 0 || i <= K || i >= n - K; }
    __host__ __device__ __forceinline__ int compact(int i) const { return (K < 0 || i <= K) ? i : i - (n - 2 * K - 1); }
    __host__ __device__ __forceinline__ int expand(int c) const { return (K < 0 || c <= K) ? c : c + (n - 2 * K - 1); }
    __host__ __device__ __forceinline__ int count() const { return K < 0 ? n : 2 * K + 1; }
};

struct PassSpec {
    long long s_row, s_out;    // source strides (elements) of row and outer index
    long long d_row, d_out;    // destination strides
    KeepMap row_in;            // rows loaded (the others are zero)
    int row_in_compact;        // loaded rows addressed by their compact index
    KeepMap row_out;           // rows stored
    int row_out_compact;       // stored rows addressed by their compact index
    KeepMap outer;             // outer indices visited (compact enumeration)
    int outer_in_compact;      // source outer index compact (else the expanded index)
    int outer_out_compact;     // destination outer index compact
    int ncols;                 // valid source columns (the others read as zero)
    int out_ncols;             // destination columns stored
    int ncolblk;               // column blocks per outer index
    int nin;                   // input fields; work items = nin * outer.count() * ncolblk
    int n_row, n_out, n_col;   // axis lengths for the wavenumbers (n_out = 0: outer is physical)
    double dk_row, dk_out, dk_col;
    double kmax2;
    int mask;                  // apply the dealias mask on load
    signed char nvar[MAXF];    // outputs per input (1 or 2)
    signed char vmul[MAXF][2]; // multiplier of each output
    signed char vout[MAXF][2]; // output field index of each output
    int nmem;                  // members of a batch (jets of one geometry in one launch), >= 1
    long long ms_in, ms_out;   // element strides between the members' inputs / outputs
};
template <typename T> struct PassPtrs {
    const V2<T> *in[MAXF];
    V2<T> *out[MAXF];
};

__host__ __device__ constexpr int pow2_floor(int v) {
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

// NB columns of 8 (FP64) or 16 (FP32) complex values make 128-byte rows;
// each thread owns E complex values of the tile; two staging buffers (the
// copy pipeline) and one buffer to transform in use at most 192 KB.
template <typename T, int N> struct PassCfg {
    static constexpr int ELEM = (int)sizeof(V2<T>);
    static constexpr int NB0 = (64 * 1024 / ELEM) / N;
    static constexpr int NB = pow2_floor(NB0 > 16 ? 16 : (NB0 < 1 ? 1 : NB0));
    static constexpr int NT0 = N * NB / 8;   // one radix-8 butterfly per thread, at most 512 threads
    static constexpr int NT = NT0 < 32 ? 32 : (NT0 > 512 ? 512 : NT0);
    static constexpr int E = N * NB / NT;
    static constexpr int TILE = N * NB;
    static constexpr bool WORK = plan_nstages(N) > 1;
    static constexpr int SMEM = (2 + (WORK ? 1 : 0)) * TILE * ELEM;
};

// Asynchronous copy of one tile (rows kept by row_in, columns < ncols; the
// rest zero-filled) into shared memory, laid out [row][NB].  Thread tid owns
// column tid % NB and rows tid / NB + k * (nt / NB).
template <typename T, int NB, int NT, int TILE>
__device__ __forceinline__ void tile_prefetch(V2<T> *dst, const V2<T> *__restrict__ src, const PassSpec &sp, int c0,
                                              int tid) {
    static_assert(NT % NB == 0, "threads must cover whole rows");
    constexpr int RSTEP = NT / NB;
    const int b = tid % NB;
    const bool col_ok = c0 + b < sp.ncols;
    const V2<T> *s = src + b;
    V2<T> *d = dst + tid;
#pragma unroll 4
    for (int row = tid / NB; row * NB < TILE; row += RSTEP, d += NT) {
        const bool ok = col_ok && sp.row_in.kept(row);
        const int r = sp.row_in_compact ? sp.row_in.compact(row) : row;
        const V2<T> *p = ok ? s + (long long)r * sp.s_row : src;
        if constexpr (sizeof(T) == 8) cp_async16(d, p, ok ? 16 : 0);
        else cp_async8(d, p, ok ? 8 : 0);
    }
}

// Persistent: block b handles items b, b + gridDim.x, ... and prefetches the
// next item's tile while transforming the current one.
template <typename T, int N, int SIGN, bool MB = false>
__global__ void __launch_bounds__(PassCfg<T, N>::NT, 1)
k_pass(const __grid_constant__ PassPtrs<T> P, const __grid_constant__ PassSpec sp, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    using C = PassCfg<T, N>;
    constexpr int NB = C::NB, NT = C::NT, TILE = C::TILE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *rawb[2] = {reinterpret_cast<V *>(smem_raw), reinterpret_cast<V *>(smem_raw) + TILE};
    V *work = reinterpret_cast<V *>(smem_raw) + 2 * TILE;
    const int tid = threadIdx.x;
    const int ntiles = sp.outer.count() * sp.ncolblk;
    const int mitems = sp.nin * ntiles;   // items of one member
    const long long nitems = MB ? (long long)sp.nmem * mitems : (long long)mitems;
    long long item = blockIdx.x;
    if (item >= nitems) return;
    // mi: member (MB: a batch of members), oc: compact outer index, o: expanded outer index
    // work items fit in 32 bits (members x inputs x outer indices x column blocks): 32-bit divisions
    auto decode = [&](long long it, int &mi, int &fi, int &oc, int &o, int &c0) {
        const int i32 = (int)it;
        mi = MB ? i32 / mitems : 0;
        const int r = MB ? i32 - mi * mitems : i32;
        fi = r / ntiles;
        const int t = r - fi * ntiles;
        oc = t / sp.ncolblk;
        o = sp.outer.expand(oc);
        c0 = (t - oc * sp.ncolblk) * NB;
    };
    auto prefetch = [&](long long it, V *dst) {
        int mi, fi, oc, o, c0;
        decode(it, mi, fi, oc, o, c0);
        const V *src = P.in[fi] + (MB ? mi * sp.ms_in : 0LL) + (long long)(sp.outer_in_compact ? oc : o) * sp.s_out + c0;
        tile_prefetch<T, NB, NT, TILE>(dst, src, sp, c0, tid);
    };
    pdl_wait();
    prefetch(item, rawb[0]);
    cp_async_commit();
    int buf = 0;
    for (; item < nitems; item += gridDim.x) {
        const long long next = item + gridDim.x;
        if (next < nitems) prefetch(next, rawb[buf ^ 1]);
        cp_async_commit();
        cp_async_wait<1>();   // this thread's copies of the current tile have landed
        __syncthreads();      // ... and everybody else's
        int mi, fi, oc, o, c0;
        decode(item, mi, fi, oc, o, c0);
        const V *cur = rawb[buf];
        const double k_out = sp.n_out ? wavenum(o, sp.n_out, sp.dk_out) : 0.0;
        const long long dbase = (MB ? mi * sp.ms_out : 0LL) + (long long)(sp.outer_out_compact ? oc : o) * sp.d_out + c0;
        const int out_cols = sp.out_ncols - c0;
        const int nv = sp.nvar[fi];
        for (int v = 0; v < nv; ++v) {
            const int mul = sp.vmul[fi][v];
            V *dst = P.out[sp.vout[fi][v]] + dbase;
            auto gld = [&](int row, int b) -> V {
                V a = cur[row * NB + b];
                if (mul == V_ONE && !sp.mask) return a;
                const double kr = wavenum(row, sp.n_row, sp.dk_row);
                const double kc = wavenum(c0 + b, sp.n_col, sp.dk_col);
                const double k2 = ksq3(kr, k_out, kc);
                if (sp.mask && k2 > sp.kmax2) return V{T(0), T(0)};   // dealias mask (solver.cu:36)
                switch (mul) {
                    case V_IK_ROW: return V{(T)(-kr) * a.y, (T)kr * a.x};
                    case V_IK_OUT: return V{(T)(-k_out) * a.y, (T)k_out * a.x};
                    case V_IK_COL: return V{(T)(-kc) * a.y, (T)kc * a.x};
                    case V_LAP: return V{(T)(-k2) * a.x, (T)(-k2) * a.y};
                    default: return a;
                }
            };
            auto gst = [&](int row, int b, V val) {
                if (b < out_cols && sp.row_out.kept(row)) {
                    const int r = sp.row_out_compact ? sp.row_out.compact(row) : row;
                    dst[(long long)r * sp.d_row + b] = val;
                }
            };
            auto smacc = [&](int row, int b) -> V & { return work[row * NB + b]; };
            fft_columns<T, N, SIGN, NB, NT>(tid, tw, gld, smacc, gst, SyncBlock{});
            __syncthreads();   // work buffer (and, after the last output, the tile buffer) free again
        }
        buf ^= 1;
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------ z pass
// One warp per pair of contiguous lines (la, la+1) of one field; 8 warps per
// block.  DIR < 0: real padded lines -> nz2 complex per line (R2C, in place).
// DIR > 0: nz2 complex -> real padded lines scaled by `scale` (C2R, in place);
// the imaginary parts of the kz = 0 and kz = nz/2 entries are ignored and the
// two padding reals of each line are set to zero.
constexpr int ZWARPS = 8;

template <typename T, int N> struct ZCfg {
    static constexpr int LEN = padded_len<T>(N);
    static constexpr int SMEM = ZWARPS * LEN * (int)sizeof(V2<T>);
};

// In-place FFT of one padded line in shared memory by one warp.
template <typename T, int N, int SIGN, int S = 0>
__device__ __forceinline__ void warp_line_fft(int lane, V2<T> *line, const V2<T> *tw) {
    using V = V2<T>;
    if constexpr (S < plan_nstages(N)) {
        fft_stage<T, N, S, SIGN, 1, 32, true>(
            lane, tw, [&](int row, int) -> V { return line[padded<T>(row)]; },
            [&](int row, int, V v) { line[padded<T>(row)] = v; }, SyncWarp{});
        __syncwarp();
        warp_line_fft<T, N, SIGN, S + 1>(lane, line, tw);
    }
}

// FFT of one padded line by one warp, ping-ponging between two line buffers
// (a and b): stage s reads one and writes the other, so a lane holds one
// radix-R butterfly at a time.  The result is in b after an odd number of
// stages and in a after an even number (see pp_result).
template <typename T, int N, int SIGN, int S = 0>
__device__ __forceinline__ void warp_line_fft_pp(int lane, V2<T> *a, V2<T> *b, const V2<T> *tw) {
    using V = V2<T>;
    if constexpr (S < plan_nstages(N)) {
        V *src = (S % 2 == 0) ? a : b;
        V *dst = (S % 2 == 0) ? b : a;
        fft_stage_stream<T, N, S, SIGN, 1, 32>(
            lane, tw, [&](int row, int) -> V { return src[padded<T>(row)]; },
            [&](int row, int, V v) { dst[padded<T>(row)] = v; });
        __syncwarp();
        warp_line_fft_pp<T, N, SIGN, S + 1>(lane, a, b, tw);
    }
}
template <typename T, int N> __host__ __device__ constexpr bool pp_result_in_b() { return plan_nstages(N) % 2 == 1; }

// In-place FFT of one padded line by the 64 threads of a warp pair that
// synchronise on named barrier `bar` (t64 = 0..63).
template <typename T, int N, int SIGN, int S = 0>
__device__ __forceinline__ void pair_line_fft(int t64, V2<T> *line, const V2<T> *tw, int bar) {
    using V = V2<T>;
    if constexpr (S < plan_nstages(N)) {
        const SyncNamed sync{bar, 64};
        fft_stage<T, N, S, SIGN, 1, 64, true>(
            t64, tw, [&](int row, int) -> V { return line[padded<T>(row)]; },
            [&](int row, int, V v) { line[padded<T>(row)] = v; }, sync);
        sync();
        pair_line_fft<T, N, SIGN, S + 1>(t64, line, tw, bar);
    }
}

// Z_k = A_k + i B_k for k <= N/2 and Z_{N-k} = conj(A_k) + i conj(B_k), from
// the half spectra of two real lines (C2R packing); Im of A_0, B_0, A_{N/2},
// B_{N/2} ignored.
template <typename T, int N>
__device__ __forceinline__ void pack_c2r(int lane, V2<T> *line, const V2<T> *__restrict__ A, const V2<T> *__restrict__ B,
                                         bool hasB) {
    using V = V2<T>;
    for (int k = lane; k <= N / 2; k += 32) {
        V a = A[k];
        V b = hasB ? B[k] : V{T(0), T(0)};
        if (k == 0 || 2 * k == N) { a.y = T(0); b.y = T(0); }
        line[padded<T>(k)] = V{a.x - b.y, a.y + b.x};
        if (k > 0 && 2 * k < N) line[padded<T>(N - k)] = V{a.x + b.y, b.x - a.y};
    }
}

// A_k = (Z_k + conj Z_{N-k})/2, B_k = (Z_k - conj Z_{N-k})/(2i), k = 0..N/2.
template <typename T, int N>
__device__ __forceinline__ void unpack_r2c(int lane, const V2<T> *line, V2<T> *__restrict__ A, V2<T> *__restrict__ B,
                                           bool hasB) {
    using V = V2<T>;
    for (int k = lane; k <= N / 2; k += 32) {
        V zk = line[padded<T>(k)];
        V zm = line[padded<T>((N - k) % N)];
        A[k] = V{T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y)};
        if (hasB) B[k] = V{T(0.5) * (zk.y + zm.y), T(-0.5) * (zk.x - zm.x)};
    }
}

template <typename T, int N, int DIR>
__global__ void __launch_bounds__(ZWARPS * 32, 2)
k_zpass(FieldSet<T> f, long long nlines, int nz2, T scale, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    V *line = reinterpret_cast<V *>(smem_raw) + warp * ZCfg<T, N>::LEN;
    const long long pair = (long long)blockIdx.x * ZWARPS + warp;
    const long long la = 2 * pair, lb = la + 1;
    if (la >= nlines) return;
    const bool hasB = lb < nlines;
    V *base = f.p[blockIdx.y];
    if constexpr (DIR < 0) {
        const T *ra = reinterpret_cast<const T *>(base + la * nz2);
        const T *rb = reinterpret_cast<const T *>(base + lb * nz2);
        for (int n = lane; n < N; n += 32) line[padded<T>(n)] = V{ra[n], hasB ? rb[n] : T(0)};
        __syncwarp();
        warp_line_fft<T, N, -1>(lane, line, tw);
        unpack_r2c<T, N>(lane, line, base + la * nz2, base + lb * nz2, hasB);
    } else {
        pack_c2r<T, N>(lane, line, base + la * nz2, base + lb * nz2, hasB);
        __syncwarp();
        warp_line_fft<T, N, +1>(lane, line, tw);
        T *ra = reinterpret_cast<T *>(base + la * nz2);
        T *rb = reinterpret_cast<T *>(base + lb * nz2);
        for (int n = lane; n < 2 * nz2; n += 32) {
            V z = n < N ? line[padded<T>(n)] : V{T(0), T(0)};
            ra[n] = z.x * scale;
            if (hasB) rb[n] = z.y * scale;
        }
    }
}

// ------------------------------------------------------------ fused z + products
// Inputs (in f.p, [x][y][kz] lines after the x and y inverse passes):
//   0 u, 1 v, 2 w, 3 w1, 4 w2, 5 w3, 6 sx, 7 sy, 8 sz,
//   [9 cx, 10 cy, 11 cz]            when two scalars,
//   [12 c, 13 lap s]                when two scalars and alpha != 0.
// Outputs written in place into f.p[0..nout): z R2C of
//   0 (w x u)_x, 1 (w x u)_y, 2 (w x u)_z    (crossProductKernel_mgpu, solver.cu:139-164)
//   3 u . grad s                             (dotKernel_mgpu, solver.cu:342-356)
//   4 alpha (lap s c + grad c . grad s) + u . grad c   (colloidAdvectionKernel_mgpu, solver.cu:374-388)
// One warp per input field; one block per line pair.
//
// Batches (the MB instantiations): the line pairs of nmem members of one
// geometry are numbered member after member (mpairs per member), and a
// member's fields lie ms elements after the previous member's; pair p of the
// batch starts at element pair_offset(p) of each field pointer.  The batch
// holds fewer than 2^31 pairs.
template <bool MB>
__device__ __forceinline__ long long pair_offset(long long p, long long mpairs, long long ms, int rawf) {
    if constexpr (MB) {
        const int pi = (int)p, mp = (int)mpairs;
        const int mi = pi / mp;
        return mi * ms + (long long)(pi - mi * mp) * rawf;
    } else {
        return p * rawf;
    }
}

template <typename T, int N> struct ZPCfg {
    static constexpr int LEN = padded_len<T>(N);   // padded line in the work area
    // work area: one bank of nph lines, or two banks when the transforms ping-pong
    __host__ __device__ static constexpr int work_bytes(int nph, bool pp) {
        return ((pp ? 2 : 1) * nph * LEN * (int)sizeof(V2<T>) + 127) / 128 * 128;
    }
    // staging area: nraw fields x a line pair of ncp complex values each
    __host__ __device__ static constexpr int pipe_bytes(int nph, int nraw, int ncp, bool pp) {
        return work_bytes(nph, pp) + nraw * 2 * ncp * (int)sizeof(V2<T>) + 16;
    }
    static constexpr int SMEM_MAX = 227 * 1024;
};

// A physical quantity of the z pass is +-raw[r0] (times i kz) +- raw[r1]
// (times i kz): the kz factors and the two-field combinations of the
// vorticity are formed here, from the lines already on chip.
struct ZRecipe { signed char r[2]; signed char ikz[2]; signed char sgn[2]; signed char pad[2]; };
struct ZRecipeSet { ZRecipe q[MAXF]; };

// C2R packing (see pack_c2r) of a combination of two raw line pairs: a
// line pair is 2*ncp complex values (line a then line b), of which the first
// nkz of each line are the kept modes (the rest of the half spectrum is zero).
template <typename T, int N>
__device__ __forceinline__ void pack_c2r_combo(int lane, V2<T> *line, const ZRecipe rc, const V2<T> *a0, const V2<T> *a1,
                                               int ncp, int nkz, double dkz) {
    using V = V2<T>;
    for (int k = lane; k <= N / 2; k += 32) {
        V a = V{T(0), T(0)}, b = V{T(0), T(0)};
        if (k < nkz) {
            const T kz = (T)wavenum(k, N, dkz);
            a = a0[k];
            b = a0[ncp + k];
            if (rc.ikz[0]) { a = V{-kz * a.y, kz * a.x}; b = V{-kz * b.y, kz * b.x}; }
            if (rc.sgn[0] < 0) { a = V{-a.x, -a.y}; b = V{-b.x, -b.y}; }
            if (a1) {
                V c = a1[k], d = a1[ncp + k];
                if (rc.ikz[1]) { c = V{-kz * c.y, kz * c.x}; d = V{-kz * d.y, kz * d.x}; }
                if (rc.sgn[1] < 0) { a = csub(a, c); b = csub(b, d); }
                else { a = cadd(a, c); b = cadd(b, d); }
            }
            if (k == 0 || 2 * k == N) { a.y = T(0); b.y = T(0); }
        }
        line[padded<T>(k)] = V{a.x - b.y, a.y + b.x};
        if (k > 0 && 2 * k < N) line[padded<T>(N - k)] = V{a.x + b.y, b.x - a.y};
    }
}

// R2C unpacking into a line pair of stride ncp: modes k <= N/2 are written,
// columns beyond N/2 (padding of short lines) are set to zero.  Threads
// t, t + nt, ... of the group share the work.
template <typename T, int N>
__device__ __forceinline__ void unpack_r2c_pad(int t, int nt, const V2<T> *line, V2<T> *A, V2<T> *B, int ncp) {
    using V = V2<T>;
    for (int k = t; k < ncp; k += nt) {
        if (k <= N / 2) {
            V zk = line[padded<T>(k)];
            V zm = line[padded<T>((N - k) % N)];
            A[k] = V{T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y)};
            B[k] = V{T(0.5) * (zk.y + zm.y), T(-0.5) * (zk.x - zm.x)};
        } else {
            A[k] = V{T(0), T(0)};
            B[k] = V{T(0), T(0)};
        }
    }
}

// Pointwise products of one line pair held in the work area (real part =
// line a, imaginary part = line b); results go to regions 0..4 of `out`
// (which may be the input bank: each point is read before it is written).
// Regions: 0 u, 1 v, 2 w, 3 w1, 4 w2, 5 w3, 6 sx, 7 sy, 8 sz,
// [9 cx, 10 cy, 11 cz], [12 c, 13 lap s].
template <typename T, int N, int NPH>
__device__ __forceinline__ void zphys_products(const V2<T> *reg, V2<T> *out, T scale, T alpha) {
    using V = V2<T>;
    constexpr int LEN = ZPCfg<T, N>::LEN;
    constexpr bool has_c = NPH >= 12, has_al = NPH >= 14;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const int pn = padded<T>(n);
        V u = reg[0 * LEN + pn], v = reg[1 * LEN + pn], w = reg[2 * LEN + pn];
        V o1 = reg[3 * LEN + pn], o2 = reg[4 * LEN + pn], o3 = reg[5 * LEN + pn];
        V sx = reg[6 * LEN + pn], sy = reg[7 * LEN + pn], sz = reg[8 * LEN + pn];
        u = cscale(u, scale); v = cscale(v, scale); w = cscale(w, scale);
        o1 = cscale(o1, scale); o2 = cscale(o2, scale); o3 = cscale(o3, scale);
        sx = cscale(sx, scale); sy = cscale(sy, scale); sz = cscale(sz, scale);
        // omega x u (crossProductKernel_mgpu, solver.cu:139-164), u . grad s (dotKernel_mgpu, :342-356)
        V n1 = V{o2.x * w.x - o3.x * v.x, o2.y * w.y - o3.y * v.y};
        V n2 = V{-o1.x * w.x + o3.x * u.x, -o1.y * w.y + o3.y * u.y};
        V n3 = V{o1.x * v.x - o2.x * u.x, o1.y * v.y - o2.y * u.y};
        V ns = V{u.x * sx.x + v.x * sy.x + w.x * sz.x, u.y * sx.y + v.y * sy.y + w.y * sz.y};
        V nc = V{T(0), T(0)};
        if constexpr (has_c) {
            // colloidAdvectionKernel_mgpu (solver.cu:374-388)
            V cx = cscale(reg[9 * LEN + pn], scale), cy = cscale(reg[10 * LEN + pn], scale);
            V cz = cscale(reg[11 * LEN + pn], scale);
            V adv = V{u.x * cx.x + v.x * cy.x + w.x * cz.x, u.y * cx.y + v.y * cy.y + w.y * cz.y};
            if constexpr (has_al) {
                V cc = cscale(reg[12 * LEN + pn], scale), ls = cscale(reg[13 * LEN + pn], scale);
                V dr = V{ls.x * cc.x + cx.x * sx.x + cy.x * sy.x + cz.x * sz.x,
                         ls.y * cc.y + cx.y * sx.y + cy.y * sy.y + cz.y * sz.y};
                nc = V{alpha * dr.x + adv.x, alpha * dr.y + adv.y};
            } else {
                nc = adv;
            }
        }
        out[0 * LEN + pn] = n1;
        out[1 * LEN + pn] = n2;
        out[2 * LEN + pn] = n3;
        out[3 * LEN + pn] = ns;
        if constexpr (has_c) out[4 * LEN + pn] = nc;
    }
}

// Persistent: block b handles line pairs b, b + gridDim.x, ...  Lines are
// [x][y] rows of ncp complex values (the kept kz modes, zero-padded).  With
// `pipe` the raw lines (NRAW fields) of the next pair are fetched with
// cp.async.bulk into a staging area while the current pair is transformed,
// multiplied and written back; otherwise they are read from global memory
// directly.  Warp q forms physical quantity q; the products are z-transformed
// back and written over raw fields 0..nout-1 of the same pair.  With PP the
// line transforms ping-pong between two banks of lines (one butterfly per
// lane at a time: fewer registers, more resident warps); otherwise they run
// in place.  A wait that times out sets bit 0 of *err and the block stops.
template <typename T, int N, int NPH, int NRAW, bool PP, bool MB = false>
__global__ void __launch_bounds__(NPH * 32, (PP && sizeof(T) == 4) ? 2 : 1)
k_zphys(const __grid_constant__ FieldSet<T> f, const __grid_constant__ ZRecipeSet zr, int nout, long long npairs,
        int ncp, int nkz, int pipe, T scale, T alpha, double dkz, const V2<T> *__restrict__ tw,
        unsigned *__restrict__ err, long long mpairs, long long ms) {
    using V = V2<T>;
    using C = ZPCfg<T, N>;
    constexpr int LEN = C::LEN;
    const int rawf = 2 * ncp;
    const unsigned raw_bytes = (unsigned)(rawf * sizeof(V));
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *bankA = reinterpret_cast<V *>(smem_raw);
    V *bankB = bankA + NPH * LEN;
    V *raw = reinterpret_cast<V *>(smem_raw + C::work_bytes(NPH, PP));
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + C::work_bytes(NPH, PP) + NRAW * raw_bytes);
    // with PP: physical values land in bank B after an odd number of stages
    constexpr bool PHYS_B = PP && pp_result_in_b<T, N>();
    V *phys = PHYS_B ? bankB : bankA;           // physical quantities
    V *prod = PP ? (PHYS_B ? bankA : bankB) : bankA;   // products (other bank with PP)
    V *fres = PP ? (pp_result_in_b<T, N>() ? (PHYS_B ? bankB : bankA) : prod) : bankA;   // forward results
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    long long pair = blockIdx.x;
    if (pair >= npairs) return;   // uniform for the block
    if (pipe) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    pdl_wait();
    const WaitCtl wc(err);
    auto issue = [&](long long p, bool withhold = false) {
        mbar_arrive_expect_tx(bar, NRAW * raw_bytes);
        if (!withhold)
            for (int q = 0; q < NRAW; ++q) bulk_g2s(raw + q * rawf, f.p[q] + pair_offset<MB>(p, mpairs, ms, rawf), raw_bytes, bar);
    };
    if (pipe && threadIdx.x == 0) issue(pair, wc.withhold);
    unsigned parity = 0;
    V *lineA = bankA + warp * LEN;
    const ZRecipe rc = zr.q[warp];
    for (; pair < npairs; pair += gridDim.x) {
        const V *a0, *a1;
        if (pipe) {
            const bool ok = mbar_wait_bounded(bar, parity, wc.limit);
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) atomicOr(err, 1u);
                mbar_wait_bounded(bar, parity, wc.limit);   // let an overdue copy land before leaving
                return;
            }
            parity ^= 1u;
            a0 = raw + rc.r[0] * rawf;
            a1 = rc.r[1] >= 0 ? raw + rc.r[1] * rawf : nullptr;
        } else {
            a0 = f.p[rc.r[0]] + pair_offset<MB>(pair, mpairs, ms, rawf);
            a1 = rc.r[1] >= 0 ? f.p[rc.r[1]] + pair_offset<MB>(pair, mpairs, ms, rawf) : nullptr;
        }
        pack_c2r_combo<T, N>(lane, lineA, rc, a0, a1, ncp, nkz, dkz);
        __syncthreads();   // staging area (or the raw lines in global memory) consumed
        if (pipe) {
            const long long next = pair + gridDim.x;
            if (threadIdx.x == 0 && next < npairs) {
                fence_proxy_async_smem();
                issue(next);
            }
        }
        __syncwarp();
        if constexpr (PP) warp_line_fft_pp<T, N, +1>(lane, lineA, bankB + warp * LEN, tw);
        else warp_line_fft<T, N, +1>(lane, lineA, tw);   // every quantity to physical space
        __syncthreads();
        zphys_products<T, N, NPH>(phys, prod, scale, alpha);
        __syncthreads();
        if (warp < nout) {   // z R2C of the products, written over raw fields 0..nout-1
            V *pl = prod + warp * LEN;
            if constexpr (PP) warp_line_fft_pp<T, N, -1>(lane, pl, (prod == bankA ? bankB : bankA) + warp * LEN, tw);
            else warp_line_fft<T, N, -1>(lane, pl, tw);
            V *d = f.p[warp] + pair_offset<MB>(pair, mpairs, ms, rawf);
            unpack_r2c_pad<T, N>(lane, 32, fres + warp * LEN, d, d + ncp, ncp);
        }
        __syncthreads();   // work area reused by the next pair
    }
}

// A spectral field holds nx ny nz2 <= 512 * 512 * 257 < 2^32 modes, so the
// index is split with 32-bit divisions.
struct SpecIdx {
    int kx, ky, kz;
    __device__ __forceinline__ SpecIdx(long long idx, const Geom &g) {
        const unsigned i = (unsigned)idx, nz2 = (unsigned)g.nz2, nx = (unsigned)g.nx;
        const unsigned t = i / nz2;
        kz = (int)(i - t * nz2);
        ky = (int)(t / nx);
        kx = (int)(t - (unsigned)ky * nx);
    }
};

// statistics reductions (k_update with STATS, k_stats_partial, k_stats_final)
constexpr int STAT_SUMS = 6;
constexpr int STAT_BLOCKS = 1184;   // 8 x 148 SMs
constexpr int STAT_THREADS = 256;

// ------------------------------------------------------------ spectral update
struct UpdCoef {
    int nf;           // fields updated: 3 + n_scalars
    int scheme;       // GNSS_SCHEME_*
    int euler;        // CN/AB2: first step
    double dt;
    double hnum[5];   // CN: dt / 2 / num with the reference's num (Re, Re*Sc, Re*Sc_c)
    double nu[5];     // IF: diffusivity per field
    double gam, zet_next, alph;   // IF-RK3 substep coefficients
    int substep;      // IF-RK3: 0, 1, 2 (substep 0 ignores the history input)
};

// Per-member update coefficients of a batch (jets of one geometry stepped by
// one launch; Reynolds and Schmidt numbers and time steps may differ).
constexpr int MAXM = 16;
struct MemberCoef {
    double dt[MAXM];
    double hnum[MAXM][5];   // CN: dt / 2 / num
    double nu[MAXM][5];     // IF: diffusivity
    double2 *mean[MAXM];    // FP32 contexts: the member's FP64 mean-profile line (or null)
};

// One warp per (ky, kx) row of the kept box, lanes along kz.  The arithmetic
// follows makeRHS / deAlias / timestep / update (solver.cu:461-657) with the
// divisions by k^2 and by (1 + dt k^2/(2 num)) done once as reciprocals.
// Rows are enumerated in the kept box (kept ky, kept kx); nl is the compact
// [kyc][kxc][ncp] layout of the forward passes; state and hist use the
// reference layout.  Along kz the unmasked modes of a row form a prefix
// (k^2 grows with kz), so the warp stops at the first chunk of 32 that is
// masked throughout.  With full_rows the masked modes of the box (kz < nkz)
// are written as zero instead (the first step of a run: it clears whatever
// the history held there); modes outside the box are never touched.  Every
// load of a mode is issued before its first store.
//
// With `mean` (FP32 contexts), the mean-profile line kx = kz = 0 (all kept ky;
// the y profiles of initialize.cu:114-194 averaged by statistics.cu:1936-2003)
// is advanced in FP64: mean[q ny + ky] holds the FP64 state of field q and
// mean[(5 + q) ny + ky] its FP64 history.  A kept value is used when it
// rounds to the FP32 value in the field (the field was last written by this
// update); otherwise the field's own value is taken, so a state written
// anew by the caller starts from what it holds.  Both copies are written.
//
// With BATCH, the rows of nmem members follow one another (state and hist of
// member m ms_sh elements after member 0's, nl ms_nl), and member m takes its
// coefficients and mean line from mc.
//
// With STATS, the kernel also sums, over the modes it writes, the spectral
// statistics of the new state (the six sums of k_stats_partial: the full
// spectrum through the kz mirror, statistics.cu:1494-1845) and writes one row
// of STAT_SUMS partials per block to `partial`; for a state that is zero
// outside the dealiasing sphere (the precondition of the step) they equal the
// sums over the whole field.
template <typename T, int SCHEME, bool STATS, bool BATCH>
__device__ __forceinline__ void k_update_body(const FieldSet<T> &state, const FieldSet<T> &hist, const FieldSet<T> &nl,
                                              const Geom &g, KeepMap kx_keep, KeepMap ky_keep, int nkz, int ncp,
                                              const UpdCoef &c, int full_rows, double *__restrict__ partial,
                                              double2 *__restrict__ mean0, const MemberCoef *mc, int nmem,
                                              long long ms_sh, long long ms_nl) {
    using V = V2<T>;
    pdl_wait();
    pdl_trigger();
    double acc[STATS ? STAT_SUMS : 1] = {};
    const int nkx = kx_keep.count(), nky = ky_keep.count();
    const int mrows = nky * nkx;   // rows of one member
    const int nrows = mrows * nmem;
    const int lane = threadIdx.x & 31;
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const bool read_hist = (SCHEME == 0) ? !c.euler : (c.substep > 0);
    const int nf = c.nf;
    for (int brow = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); brow < nrows; brow += nwarp) {
        const int mi = BATCH ? brow / mrows : 0;
        const int row = BATCH ? brow - mi * mrows : brow;
        const int kyc = row / nkx, kxc = row - kyc * nkx;
        const int kxi = kx_keep.expand(kxc), kyi = ky_keep.expand(kyc);
        const double k1 = wavenum(kxi, g.nx, g.dkx), k2 = wavenum(kyi, g.ny, g.dky);
        const long long base = ((long long)kyi * g.nx + kxi) * g.nz2 + (BATCH ? mi * ms_sh : 0);   // state / hist
        const long long jbase = (long long)row * ncp + (BATCH ? mi * ms_nl : 0);                    // nonlinear term
        double2 *const mean = BATCH ? mc->mean[mi] : mean0;
        const double c_dt = BATCH ? mc->dt[mi] : c.dt;
        for (int k0 = 0; k0 < nkz; k0 += 32) {
            const int kzi = k0 + lane;
            const bool inrow = kzi < nkz;
            const double k3 = wavenum(kzi, g.nz, g.dkz);
            const double ksq = ksq3(k1, k2, k3);
            const bool masked = ksq > g.kmax2;
            if (!full_rows && __all_sync(0xffffffffu, masked || !inrow)) break;
            if (!inrow) continue;
            const long long idx = base + kzi, jdx = jbase + kzi;
            if (masked) {
                // deAlias of the state and of the right-hand side (solver.cu:36, 756)
                if (full_rows) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
                        if (q < nf) {
                            state.p[q][idx] = V{T(0), T(0)};
                            hist.p[q][idx] = V{T(0), T(0)};
                        }
                    }
                }
                continue;
            }
            V a[5], f[5], h[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                a[q] = V{T(0), T(0)};
                f[q] = V{T(0), T(0)};
                h[q] = V{T(0), T(0)};
                if (q < nf) {
                    a[q] = nl.p[q][jdx];
                    f[q] = state.p[q][idx];
                    if (read_hist) h[q] = hist.p[q][idx];
                }
            }
            // makeRHS: (k k^T / k^2 - I) N for the velocity, -N for the scalars,
            // zero at k = 0 (solver.cu:461-521)
            double R[5][2];
            if (kxi == 0 && kyi == 0 && kzi == 0) {
#pragma unroll
                for (int q = 0; q < 5; ++q) R[q][0] = R[q][1] = 0.0;
            } else {
                const double ik = 1.0 / ksq;
                const double pr = (k1 * (double)a[0].x + k2 * (double)a[1].x + k3 * (double)a[2].x) * ik;
                const double pi = (k1 * (double)a[0].y + k2 * (double)a[1].y + k3 * (double)a[2].y) * ik;
                R[0][0] = k1 * pr - (double)a[0].x;
                R[0][1] = k1 * pi - (double)a[0].y;
                R[1][0] = k2 * pr - (double)a[1].x;
                R[1][1] = k2 * pi - (double)a[1].y;
                R[2][0] = k3 * pr - (double)a[2].x;
                R[2][1] = k3 * pi - (double)a[2].y;
#pragma unroll
                for (int q = 3; q < 5; ++q) {
                    R[q][0] = -(double)a[q].x;
                    R[q][1] = -(double)a[q].y;
                }
            }
            V sv[STATS ? 5 : 1];   // the stored new state (the statistics read these values)
            // the mean-profile line in FP64 (FP32 contexts)
            const bool mline = sizeof(T) == 4 && mean != nullptr && kxi == 0 && kzi == 0;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                if constexpr (STATS) sv[q] = V{T(0), T(0)};
                if (q >= nf) break;
                double fr = (double)f[q].x, fi = (double)f[q].y;
                double hr = (double)h[q].x, hi = (double)h[q].y;
                if (mline) {
                    const double2 sm = mean[q * g.ny + kyi];
                    if ((T)sm.x == f[q].x && (T)sm.y == f[q].y) { fr = sm.x; fi = sm.y; }
                    if (read_hist) {
                        const double2 hm = mean[(5 + q) * g.ny + kyi];
                        if ((T)hm.x == h[q].x && (T)hm.y == h[q].y) { hr = hm.x; hi = hm.y; }
                    }
                }
                double nr, ni, gr, gi;   // new state and new history
                if constexpr (SCHEME == 0) {
                    // eulerKernel_mgpu / adamsBashforthKernel_mgpu (solver.cu:547-585)
                    const double hk = (BATCH ? mc->hnum[mi][q] : c.hnum[q]) * ksq;
                    const double am = 1.0 - hk;
                    const double ib = 1.0 / (1.0 + hk);
                    if (c.euler) {
                        nr = (am * fr + c_dt * R[q][0]) * ib;
                        ni = (am * fi + c_dt * R[q][1]) * ib;
                    } else {
                        nr = (am * fr + c_dt * (1.5 * R[q][0] - 0.5 * hr)) * ib;
                        ni = (am * fi + c_dt * (1.5 * R[q][1] - 0.5 * hi)) * ib;
                    }
                    gr = R[q][0];   // updateKernel_mgpu (solver.cu:618-637)
                    gi = R[q][1];
                } else {
                    const double E = exp(-(BATCH ? mc->nu[mi][q] : c.nu[q]) * ksq * c.alph * c_dt);
                    nr = E * (fr + c.gam * c_dt * R[q][0] + hr);
                    ni = E * (fi + c.gam * c_dt * R[q][1] + hi);
                    gr = c.zet_next * c_dt * E * R[q][0];
                    gi = c.zet_next * c_dt * E * R[q][1];
                }
                state.p[q][idx] = V{(T)nr, (T)ni};
                if constexpr (STATS) sv[q] = V{(T)nr, (T)ni};
                hist.p[q][idx] = V{(T)gr, (T)gi};
                if (mline) {
                    mean[q * g.ny + kyi] = double2{nr, ni};
                    mean[(5 + q) * g.ny + kyi] = double2{gr, gi};
                }
            }
            if constexpr (STATS) {   // sums of the stored (T) values, as k_stats_partial reads them
                const double wt = (kzi == 0 || 2 * kzi == g.nz) ? 1.0 : 2.0;
                const bool origin = kxi == 0 && kyi == 0 && kzi == 0;
                double m[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) m[q] = (double)sv[q].x * sv[q].x + (double)sv[q].y * sv[q].y;
                const double e = m[0] + m[1] + m[2];
                acc[0] += wt * e;
                acc[1] += wt * ksq * e;
                acc[2] += wt * ksq * m[3];
                acc[3] += wt * ksq * m[4];
                if (!origin) {
                    acc[4] += wt * m[3];
                    acc[5] += wt * m[4];
                }
            }
        }
    }
    if constexpr (STATS) {   // fixed-order block reduction: warp shuffles, then the block's warps in order
        __shared__ double red[STAT_SUMS][8];
#pragma unroll
        for (int q = 0; q < STAT_SUMS; ++q) {
            double v = acc[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[q][threadIdx.x >> 5] = v;
        }
        __syncthreads();
        if (threadIdx.x < STAT_SUMS) {
            double v = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
            partial[blockIdx.x * STAT_SUMS + threadIdx.x] = v;
        }
    }
}

template <typename T, int SCHEME, bool STATS = false, bool BATCH = false>
__global__ void __launch_bounds__(256)
k_update(const __grid_constant__ FieldSet<T> state, const __grid_constant__ FieldSet<T> hist,
         const __grid_constant__ FieldSet<T> nl, Geom g, KeepMap kx_keep, KeepMap ky_keep, int nkz, int ncp,
         UpdCoef c, int full_rows, double *__restrict__ partial = nullptr, double2 *__restrict__ mean = nullptr) {
    k_update_body<T, SCHEME, STATS, false>(state, hist, nl, g, kx_keep, ky_keep, nkz, ncp, c, full_rows, partial,
                                           mean, nullptr, 1, 0, 0);
}
template <typename T, int SCHEME>
__global__ void __launch_bounds__(256)
k_update_batch(const __grid_constant__ FieldSet<T> state, const __grid_constant__ FieldSet<T> hist,
               const __grid_constant__ FieldSet<T> nl, Geom g, KeepMap kx_keep, KeepMap ky_keep, int nkz, int ncp,
               UpdCoef c, int full_rows, const __grid_constant__ MemberCoef mc, int nmem, long long ms_sh,
               long long ms_nl) {
    k_update_body<T, SCHEME, false, true>(state, hist, nl, g, kx_keep, ky_keep, nkz, ncp, c, full_rows, nullptr,
                                          nullptr, &mc, nmem, ms_sh, ms_nl);
}

// ------------------------------------------------------------ statistics
// Six sums per thread, Kahan-compensated, reduced in a fixed tree order per
// block; the partials are summed in a fixed order by one block.  The result
// is independent of scheduling (unlike atomicAdd in statistics.cu:1555).

struct Kahan {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        double y = x - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

template <typename T>
__global__ void __launch_bounds__(STAT_THREADS)
k_stats_partial(FieldSet<T> st, int has_s, int has_c, Geom g, double *__restrict__ partial) {
    using V = V2<T>;
    __shared__ double red[STAT_SUMS][STAT_THREADS];
    Kahan acc[STAT_SUMS];
    const long long nspec = (long long)g.nx * g.ny * g.nz2;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nspec;
         idx += (long long)gridDim.x * blockDim.x) {
        const SpecIdx si(idx, g);
        const int kzi = si.kz, kxi = si.kx, kyi = si.ky;
        const double k1 = wavenum(kxi, g.nx, g.dkx), k2 = wavenum(kyi, g.ny, g.dky), k3 = wavenum(kzi, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const double wt = (kzi == 0 || 2 * kzi == g.nz) ? 1.0 : 2.0;   // kz mirror (statistics.cu:1505-1532)
        V a = st.p[0][idx], b = st.p[1][idx], c = st.p[2][idx];
        const double e = (double)a.x * a.x + (double)a.y * a.y + (double)b.x * b.x + (double)b.y * b.y +
                         (double)c.x * c.x + (double)c.y * c.y;
        acc[0].add(wt * e);
        acc[1].add(wt * ksq * e);
        const bool k0 = (idx == 0);
        if (has_s) {
            V s = st.p[3][idx];
            const double m = (double)s.x * s.x + (double)s.y * s.y;
            acc[2].add(wt * ksq * m);
            if (!k0) acc[4].add(wt * m);
        }
        if (has_c) {
            V s = st.p[4][idx];
            const double m = (double)s.x * s.x + (double)s.y * s.y;
            acc[3].add(wt * ksq * m);
            if (!k0) acc[5].add(wt * m);
        }
    }
    for (int q = 0; q < STAT_SUMS; ++q) red[q][threadIdx.x] = acc[q].s;
    __syncthreads();
    for (int w = STAT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < STAT_SUMS; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < STAT_SUMS; ++q) partial[blockIdx.x * STAT_SUMS + q] = red[q][0];
}

__global__ void __launch_bounds__(STAT_SUMS * 32) k_stats_final(const double *__restrict__ partial, int nblocks,
                                                                 double *__restrict__ out) {
    // warp q sums column q: lanes stride the blocks, then a fixed shuffle tree
    pdl_wait();
    pdl_trigger();
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Kahan acc;
    for (int b = lane; b < nblocks; b += 32) acc.add(partial[b * STAT_SUMS + q]);
    double v = acc.s;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[q] = v;
}

// ------------------------------------------------------------ reference-surface ops
// Spectral index helpers for the transposed layout idx = kz + nz2*(x + nx*y).
#define GNSS_GRID_STRIDE(n) \
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < (n); idx += (long long)gridDim.x * blockDim.x)

template <typename T> __global__ void k_dealias(V2<T> *f, Geom g) {
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        if (ksq3(k1, k2, k3) > g.kmax2) f[idx] = V2<T>{T(0), T(0)};
    }
}

// The reference's solver_ps takes the velocity through an inverse and a
// forward transform before the vorticity and the time step use it
// (solver.cu:707-722, :743-750).  The complex-to-real z transform of that
// round trip keeps the Hermitian part of the kz = 0 and kz = nz/2 planes,
// F(k) -> (F(k) + conj F(-k)) / 2.  The velocity of a state departs from
// that symmetry only at kept Nyquist modes: makeRHS (solver.cu:461-521)
// projects a Nyquist mode and its mirror with the same wavenumber -n/2, so
// the projected right-hand side there is not Hermitian.  k_herm applies the
// round trip's projection to u, v, w where that can happen:
//   in the kz = 0 plane, the ky Nyquist row (row_y) and the kx Nyquist
//   column (col_x), mirror (-kx, -ky);
//   the whole kz = nz/2 plane (plane_z), mirror (-kx, -ky).
// One thread per pair of mirror modes (a mode that is its own mirror keeps
// its real part).  In FP32 contexts the FP64 mean-profile entry of the ky
// Nyquist row (mc.mean[member]) gets the same treatment.  Members of a batch
// are ms elements apart.
template <typename T>
__global__ void k_herm(FieldSet<T> f, Geom g, int row_y, int col_x, int plane_z, const __grid_constant__ MemberCoef mc,
                       int nmem, long long ms) {
    using V = V2<T>;
    pdl_wait();
    pdl_trigger();
    const int nx = g.nx, ny = g.ny;
    const long long na = row_y ? nx : 0, nb = col_x ? ny : 0, nc = plane_z ? (long long)nx * ny : 0;
    const long long per = na + nb + nc;
    GNSS_GRID_STRIDE(per * nmem) {
        const int mi = (int)(idx / per);
        long long t = idx - (long long)mi * per;
        int i, j, kz;
        if (t < na) {   // kz = 0, ky Nyquist row
            i = (int)t; j = ny / 2; kz = 0;
        } else if ((t -= na) < nb) {   // kz = 0, kx Nyquist column (its ky Nyquist entry belongs to the row)
            i = nx / 2; j = (int)t; kz = 0;
            if (row_y && j == ny / 2) continue;
        } else {   // kz = nz/2 plane
            t -= nb;
            j = (int)(t / nx); i = (int)(t - (long long)j * nx); kz = g.nz / 2;
        }
        const int mi2 = (nx - i) % nx, mj2 = (ny - j) % ny;
        if ((long long)mj2 * nx + mi2 < (long long)j * nx + i) continue;   // the pair is done from its other mode
        const long long a = ((long long)j * nx + i) * g.nz2 + kz + (long long)mi * ms;
        const long long b = ((long long)mj2 * nx + mi2) * g.nz2 + kz + (long long)mi * ms;
        double2 *const mean = mc.mean[mi];
        for (int q = 0; q < 3; ++q) {
            const V x = f.p[q][a], y = f.p[q][b];
            const V h = V{T(0.5) * (x.x + y.x), T(0.5) * (x.y - y.y)};
            f.p[q][a] = h;
            f.p[q][b] = V{h.x, -h.y};
            if (mean && kz == 0 && i == 0 && a == b) mean[q * ny + j].y = 0.0;   // the FP64 mean-profile entry
        }
    }
}

template <typename T>
__global__ void k_vorticity(const V2<T> *u, const V2<T> *v, const V2<T> *w, V2<T> *o1, V2<T> *o2, V2<T> *o3, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = u[idx], b = v[idx], c = w[idx];
        o1[idx] = V{-k2 * c.y + k3 * b.y, k2 * c.x - k3 * b.x};
        o2[idx] = V{k1 * c.y - k3 * a.y, -k1 * c.x + k3 * a.x};
        o3[idx] = V{-k1 * b.y + k2 * a.y, k1 * b.x - k2 * a.x};
    }
}

template <typename T> __global__ void k_gradient(const V2<T> *f, V2<T> *fx, V2<T> *fy, V2<T> *fz, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = f[idx];
        fx[idx] = V{-k1 * a.y, k1 * a.x};
        fy[idx] = V{-k2 * a.y, k2 * a.x};
        fz[idx] = V{-k3 * a.y, k3 * a.x};
    }
}

template <typename T>
__global__ void k_divergence(const V2<T> *fx, const V2<T> *fy, const V2<T> *fz, V2<T> *out, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = fx[idx], b = fy[idx], c = fz[idx];
        out[idx] = V{-k1 * a.y - k2 * b.y - k3 * c.y, k1 * a.x + k2 * b.x + k3 * c.x};
    }
}

template <typename T>
__global__ void k_make_rhs(V2<T> *ru, V2<T> *rv, V2<T> *rw, V2<T> *rs, V2<T> *rc, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        if (s.kx == 0 && s.ky == 0 && s.kz == 0) {
            ru[idx] = rv[idx] = rw[idx] = V{T(0), T(0)};
            if (rs) rs[idx] = V{T(0), T(0)};
            if (rc) rc[idx] = V{T(0), T(0)};
            continue;
        }
        V a = ru[idx], b = rv[idx], c = rw[idx];
        double t1r = a.x, t1c = a.y, t2r = b.x, t2c = b.y, t3r = c.x, t3c = c.y;
        ru[idx] = V{(T)((k1 * k1 / ksq - 1.0) * t1r + (k1 * k2 / ksq) * t2r + (k1 * k3 / ksq) * t3r),
                    (T)((k1 * k1 / ksq - 1.0) * t1c + (k1 * k2 / ksq) * t2c + (k1 * k3 / ksq) * t3c)};
        rv[idx] = V{(T)((k2 * k1 / ksq) * t1r + (k2 * k2 / ksq - 1.0) * t2r + (k2 * k3 / ksq) * t3r),
                    (T)((k2 * k1 / ksq) * t1c + (k2 * k2 / ksq - 1.0) * t2c + (k2 * k3 / ksq) * t3c)};
        rw[idx] = V{(T)((k3 * k1 / ksq) * t1r + (k3 * k2 / ksq) * t2r + (k3 * k3 / ksq - 1.0) * t3r),
                    (T)((k3 * k1 / ksq) * t1c + (k3 * k2 / ksq) * t2c + (k3 * k3 / ksq - 1.0) * t3c)};
        if (rs) { V q = rs[idx]; rs[idx] = V{-q.x, -q.y}; }
        if (rc) { V q = rc[idx]; rc[idx] = V{-q.x, -q.y}; }
    }
}

template <typename T>
__global__ void k_timestep(V2<T> *f, const V2<T> *r, const V2<T> *ro, double num, double dt, int euler, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const double a = 1.0 - dt / 2.0 * ksq / num, b = 1.0 + dt / 2.0 * ksq / num;
        V fv = f[idx], rv = r[idx];
        double nr, ni;
        if (euler) {
            nr = (a * fv.x + dt * rv.x) / b;
            ni = (a * fv.y + dt * rv.y) / b;
        } else {
            V o = ro[idx];
            nr = (a * fv.x + dt * (1.5 * rv.x - 0.5 * o.x)) / b;
            ni = (a * fv.y + dt * (1.5 * rv.y - 0.5 * o.y)) / b;
        }
        f[idx] = V{(T)nr, (T)ni};
    }
}

template <typename T> __global__ void k_shift_history(V2<T> *r, V2<T> *ro, long long ns) {
    GNSS_GRID_STRIDE(ns) {
        ro[idx] = r[idx];
        r[idx] = V2<T>{T(0), T(0)};
    }
}

// physical-space point loop over x < nx, y < ny, z < nz of the padded layout
// (nx ny nz <= 512^3 < 2^32 points: 32-bit divisions)
struct PhysIdx {
    long long p;
    __device__ __forceinline__ PhysIdx(long long idx, const Geom &g) {
        const unsigned i = (unsigned)idx, nz = (unsigned)g.nz, ny = (unsigned)g.ny;
        const unsigned t = i / nz;
        const int z = (int)(i - t * nz);
        const unsigned x = t / ny;
        const int y = (int)(t - x * ny);
        p = (long long)z + 2LL * g.nz2 * ((long long)y + (long long)g.ny * (long long)x);
    }
};

template <typename T>
__global__ void k_cross(const T *u, const T *v, const T *w, T *o1, T *o2, T *o3, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        const T w1 = o1[p], w2 = o2[p], w3 = o3[p];
        o1[p] = w2 * w[p] - w3 * v[p];
        o2[p] = -w1 * w[p] + w3 * u[p];
        o3[p] = w1 * v[p] - w2 * u[p];
    }
}

template <typename T>
__global__ void k_dot(const T *a1, const T *a2, const T *a3, const T *b1, const T *b2, const T *b3, T *out, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        out[p] = a1[p] * b1[p] + a2[p] * b2[p] + a3[p] * b3[p];
    }
}

template <typename T>
__global__ void k_colloid(const T *u, const T *v, const T *w, const T *c, const T *cx, const T *cy, const T *cz,
                          const T *sx, const T *sy, const T *sz, T *lap, T alpha, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        lap[p] = alpha * (lap[p] * c[p] + cx[p] * sx[p] + cy[p] * sy[p] + cz[p] * sz[p]) + u[p] * cx[p] +
                 v[p] * cy[p] + w[p] * cz[p];
    }
}

}  // namespace gnss

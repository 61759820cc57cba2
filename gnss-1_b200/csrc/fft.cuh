// fft.cuh -- device FFT building blocks for the B200 pseudospectral step.
//
// Stockham autosort FFT (mixed radix 8/4/2/3) executed cooperatively by a
// thread block (strided "tile" passes over x and y) or by one warp (one
// contiguous z line pair).  A stage with radix R and span NS takes butterfly
// jj in [0, N/R), reads rows jj + r*N/R, multiplies row r by the twiddle
// W_N^(r*(jj%NS)*N/(NS*R)), does a length-R DFT in registers and writes rows
// (jj/NS)*NS*R + jj%NS + r*NS.  The first stage reads rows jj + r*N/R and the
// last stage writes rows jj + r*N/R, so both can talk to global memory
// directly with coalesced row accesses while the middle stages exchange data
// through shared memory.
//
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / N) (computed
// on the host in long double); SIGN = +1 (inverse) uses conj(tw).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gnss {

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };
template <typename T> using V2 = typename Vec2<T>::type;

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    return V{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) {
    return V{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
// (S * i) * a
template <int S, typename V> __device__ __forceinline__ V mul_si(V a) {
    return S > 0 ? V{-a.y, a.x} : V{a.y, -a.x};
}
template <typename V, typename T> __device__ __forceinline__ V cscale(V a, T s) { return V{a.x * s, a.y * s}; }

// ------------------------------------------------------------ radix plans
// Greedy plan: radix 8 while possible, then 4, 2, and finally 3s.
__host__ __device__ constexpr int plan_radix(int n, int s) {
    int rem = n, st = 0;
    while (rem > 1) {
        int r = (rem % 8 == 0) ? 8 : (rem % 4 == 0) ? 4 : (rem % 2 == 0) ? 2 : (rem % 3 == 0) ? 3 : -1;
        if (r < 0) return -1;
        if (st == s) return r;
        rem /= r;
        ++st;
    }
    return 1;
}
__host__ __device__ constexpr int plan_nstages(int n) {
    int st = 0;
    while (plan_radix(n, st) > 1) ++st;
    return st;
}
__host__ __device__ constexpr int plan_span(int n, int s) {
    int ns = 1;
    for (int i = 0; i < s; ++i) ns *= plan_radix(n, i);
    return ns;
}
__host__ __device__ constexpr bool plan_ok(int n) {
    for (int s = 0; s < 16; ++s) {
        int r = plan_radix(n, s);
        if (r < 0) return false;
        if (r == 1) return true;
    }
    return false;
}

// ------------------------------------------------------------ small DFTs
template <int R, int S, typename V> struct Dft;

template <int S, typename V> struct Dft<2, S, V> {
    static __device__ __forceinline__ void run(V *v) {
        V t = v[0];
        v[0] = cadd(t, v[1]);
        v[1] = csub(t, v[1]);
    }
};

template <int S, typename V> struct Dft<3, S, V> {
    static __device__ __forceinline__ void run(V *v) {
        using T = decltype(v[0].x);
        const T c3 = T(-0.5);
        const T s3 = T(0.86602540378443864676372317075294);
        V s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        V m0 = V{v[0].x + c3 * s.x, v[0].y + c3 * s.y};
        V jd = mul_si<S>(V{s3 * d.x, s3 * d.y});
        v[0] = cadd(v[0], s);
        v[1] = cadd(m0, jd);
        v[2] = csub(m0, jd);
    }
};

template <int S, typename V> __device__ __forceinline__ void dft4(V &a0, V &a1, V &a2, V &a3) {
    V s02 = cadd(a0, a2), d02 = csub(a0, a2);
    V s13 = cadd(a1, a3), d13 = mul_si<S>(csub(a1, a3));
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, d13);
    a3 = csub(d02, d13);
}

template <int S, typename V> struct Dft<4, S, V> {
    static __device__ __forceinline__ void run(V *v) { dft4<S>(v[0], v[1], v[2], v[3]); }
};

template <int S, typename V> struct Dft<8, S, V> {
    static __device__ __forceinline__ void run(V *v) {
        using T = decltype(v[0].x);
        const T h = T(0.70710678118654752440084436210485);
        V e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        V o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<S>(e0, e1, e2, e3);
        dft4<S>(o0, o1, o2, o3);
        // o1 *= (1 + S i)/sqrt2 ; o2 *= S i ; o3 *= (-1 + S i)/sqrt2
        V t1 = V{h * (o1.x - T(S) * o1.y), h * (o1.y + T(S) * o1.x)};
        V t2 = mul_si<S>(o2);
        V t3 = V{h * (-o3.x - T(S) * o3.y), h * (-o3.y + T(S) * o3.x)};
        v[0] = cadd(e0, o0);
        v[4] = csub(e0, o0);
        v[1] = cadd(e1, t1);
        v[5] = csub(e1, t1);
        v[2] = cadd(e2, t2);
        v[6] = csub(e2, t2);
        v[3] = cadd(e3, t3);
        v[7] = csub(e3, t3);
    }
};

// ------------------------------------------------------------ one stage
// Jobs are numbered job = b + NB*jj (column b fastest) so that consecutive
// threads touch consecutive columns of a row.  LD(row, b) -> V, ST(row, b, V).
// All loads of a thread happen before any of its stores; MIDSYNC inserts the
// block/warp barrier between the two phases (needed when LD and ST address
// the same shared buffer).
struct SyncBlock { __device__ __forceinline__ void operator()() const { __syncthreads(); } };
struct SyncWarp { __device__ __forceinline__ void operator()() const { __syncwarp(); } };
struct SyncNone { __device__ __forceinline__ void operator()() const {} };
// named barrier shared by a subset of the block's warps (ids 1..15; 0 is __syncthreads)
struct SyncNamed {
    int id, nthreads;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
    }
};

template <typename T, int N, int STAGE, int SIGN, int NB, int NT, bool MIDSYNC, class LD, class ST, class SYNC>
__device__ __forceinline__ void fft_stage(int tid, const V2<T> *__restrict__ tw, LD ld, ST st, SYNC sync) {
    using V = V2<T>;
    constexpr int R = plan_radix(N, STAGE);
    constexpr int NS = plan_span(N, STAGE);
    constexpr int M = N / R;
    constexpr int NJ = M * NB;
    constexpr int PER = (NJ + NT - 1) / NT;
    constexpr int TSTEP = N / (NS * R);
    V v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int job = tid + p * NT;
        if ((NJ % NT == 0) || job < NJ) {
            const int b = job % NB, jj = job / NB;
#pragma unroll
            for (int r = 0; r < R; ++r) v[p][r] = ld(jj + r * M, b);
            if (NS > 1) {
                const int k = jj % NS;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    V w = __ldg(&tw[r * k * TSTEP]);
                    v[p][r] = (SIGN < 0) ? cmul(v[p][r], w) : cmulc(v[p][r], w);
                }
            }
            Dft<R, SIGN, V>::run(v[p]);
        }
    }
    if (MIDSYNC) sync();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int job = tid + p * NT;
        if ((NJ % NT == 0) || job < NJ) {
            const int b = job % NB, jj = job / NB;
            const int k = jj % NS;
            const int idxD = (jj / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) st(idxD + r * NS, b, v[p][r]);
        }
    }
}

// A stage whose source and destination buffers differ: each butterfly is
// stored as soon as it is computed, so a thread holds one butterfly at a time.
template <typename T, int N, int STAGE, int SIGN, int NB, int NT, class LD, class ST>
__device__ __forceinline__ void fft_stage_stream(int tid, const V2<T> *__restrict__ tw, LD ld, ST st) {
    using V = V2<T>;
    constexpr int R = plan_radix(N, STAGE);
    constexpr int NS = plan_span(N, STAGE);
    constexpr int M = N / R;
    constexpr int NJ = M * NB;
    constexpr int PER = (NJ + NT - 1) / NT;
    constexpr int TSTEP = N / (NS * R);
#pragma unroll 1
    for (int p = 0; p < PER; ++p) {
        const int job = tid + p * NT;
        if ((NJ % NT == 0) || job < NJ) {
            const int b = job % NB, jj = job / NB;
            V v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = ld(jj + r * M, b);
            if (NS > 1) {
                const int k = jj % NS;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    V w = __ldg(&tw[r * k * TSTEP]);
                    v[r] = (SIGN < 0) ? cmul(v[r], w) : cmulc(v[r], w);
                }
            }
            Dft<R, SIGN, V>::run(v);
            const int idxD = (jj / NS) * NS * R + jj % NS;
#pragma unroll
            for (int r = 0; r < R; ++r) st(idxD + r * NS, b, v[r]);
        }
    }
}

// Run stages [S0, S1) all reading and writing the shared buffer through the
// accessor SM (row, b) -> V&.  Each stage ends with a barrier.
template <typename T, int N, int S, int S1, int SIGN, int NB, int NT, class SM, class SYNC>
__device__ __forceinline__ void fft_mid_stages(int tid, const V2<T> *tw, SM sm, SYNC sync) {
    if constexpr (S < S1) {
        using V = V2<T>;
        fft_stage<T, N, S, SIGN, NB, NT, true>(
            tid, tw, [&](int row, int b) -> V { return sm(row, b); },
            [&](int row, int b, V val) { sm(row, b) = val; }, sync);
        sync();
        fft_mid_stages<T, N, S + 1, S1, SIGN, NB, NT>(tid, tw, sm, sync);
    }
}

// Full FFT of NB columns of length N: the first stage reads through GLD, the
// last writes through GST, the middle ones go through shared memory SM.
// With a single stage the data never touches shared memory.  On return all
// stores through GST have been issued; the shared buffer may be reused after
// the caller's barrier.
template <typename T, int N, int SIGN, int NB, int NT, class GLD, class SM, class GST, class SYNC>
__device__ __forceinline__ void fft_columns(int tid, const V2<T> *tw, GLD gld, SM sm, GST gst, SYNC sync) {
    using V = V2<T>;
    constexpr int NSTG = plan_nstages(N);
    static_assert(plan_ok(N), "transform length must be 2^a 3^b");
    if constexpr (NSTG == 1) {
        fft_stage<T, N, 0, SIGN, NB, NT, false>(tid, tw, gld, gst, sync);
    } else {
        fft_stage<T, N, 0, SIGN, NB, NT, false>(
            tid, tw, gld, [&](int row, int b, V val) { sm(row, b) = val; }, sync);
        sync();
        fft_mid_stages<T, N, 1, NSTG - 1, SIGN, NB, NT>(tid, tw, sm, sync);
        fft_stage<T, N, NSTG - 1, SIGN, NB, NT, false>(
            tid, tw, [&](int row, int b) -> V { return sm(row, b); }, gst, sync);
    }
}

// ---------------------------------------------------------------- stage 0 in registers
// Stage 0 (span 1, no twiddles) of a column FFT whose inputs a thread already
// holds in registers: v[p][r] is element (row jj + r*N/R, column b) of the
// thread's p-th butterfly, job = tid + p*NT, b = job % NB, jj = job / NB.
template <typename T, int N, int NB, int NT> struct Stage0 {
    static constexpr int R = plan_radix(N, 0);
    static constexpr int M = N / R;
    static constexpr int NJ = M * NB;
    static constexpr int PER = (NJ + NT - 1) / NT;
};

// v[p][r] = LD(row, b) for this thread's stage-0 elements
template <typename T, int N, int NB, int NT, class LD>
__device__ __forceinline__ void stage0_gather(int tid, V2<T> (&v)[Stage0<T, N, NB, NT>::PER][Stage0<T, N, NB, NT>::R],
                                              LD ld) {
    using S0 = Stage0<T, N, NB, NT>;
#pragma unroll
    for (int p = 0; p < S0::PER; ++p) {
        const int job = tid + p * NT;
        if ((S0::NJ % NT == 0) || job < S0::NJ) {
            const int b = job % NB, jj = job / NB;
#pragma unroll
            for (int r = 0; r < S0::R; ++r) v[p][r] = ld(jj + r * S0::M, b);
        }
    }
}

// Stage 0 from registers: MUL(value, row, b) is applied to each input
// element and the stage-0 outputs go through ST(row, b, V) (shared memory,
// or global memory when the transform has a single stage).
template <typename T, int N, int SIGN, int NB, int NT, class MUL, class ST>
__device__ __forceinline__ void stage0_from_regs(int tid,
                                                 const V2<T> (&v)[Stage0<T, N, NB, NT>::PER][Stage0<T, N, NB, NT>::R],
                                                 MUL mul, ST st) {
    using V = V2<T>;
    using S0 = Stage0<T, N, NB, NT>;
#pragma unroll
    for (int p = 0; p < S0::PER; ++p) {
        const int job = tid + p * NT;
        if ((S0::NJ % NT == 0) || job < S0::NJ) {
            const int b = job % NB, jj = job / NB;
            V w[S0::R];
#pragma unroll
            for (int r = 0; r < S0::R; ++r) w[r] = mul(v[p][r], jj + r * S0::M, b);
            Dft<S0::R, SIGN, V>::run(w);
#pragma unroll
            for (int r = 0; r < S0::R; ++r) st(jj * S0::R + r, b, w[r]);
        }
    }
}

// Stages 1 .. NSTG-1 of a column FFT whose stage-0 output is in shared
// memory (accessor SM); the last stage stores through GST.  Requires a
// barrier between stage 0's stores and this call.
template <typename T, int N, int SIGN, int NB, int NT, class SM, class GST, class SYNC>
__device__ __forceinline__ void fft_rest_stages(int tid, const V2<T> *tw, SM sm, GST gst, SYNC sync) {
    using V = V2<T>;
    constexpr int NSTG = plan_nstages(N);
    if constexpr (NSTG > 1) {
        fft_mid_stages<T, N, 1, NSTG - 1, SIGN, NB, NT>(tid, tw, sm, sync);
        fft_stage<T, N, NSTG - 1, SIGN, NB, NT, false>(
            tid, tw, [&](int row, int b) -> V { return sm(row, b); }, gst, sync);
    }
}

// Padded index for one contiguous line in shared memory: one spare element
// every 8 (double2) or 16 (float2) entries spreads the stride-8 stores of
// the radix-8 stages over the banks (measured best of the two spacings).
template <typename T> __host__ __device__ constexpr int pad_div() { return sizeof(T) == 8 ? 8 : 16; }
template <typename T> __host__ __device__ __forceinline__ constexpr int padded(int i) { return i + i / pad_div<T>(); }
template <typename T> __host__ __device__ constexpr int padded_len(int n) { return n + n / pad_div<T>() + 1; }

}  // namespace gnss

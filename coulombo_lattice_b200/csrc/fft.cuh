// Shared-memory mixed-radix FFT for sm_100a.
//
// Lines of length n sit in shared memory in "column" layout: element idx of line l is at
// buf[idx * ld + l], so consecutive threads touch consecutive lines and a warp never
// serialises on a bank.  The transform is the Stockham autosort formulation (Govindaraju et
// al., "High Performance Discrete Fourier Transforms on Graphics Processors", SC08): every
// stage of radix R reads R inputs n/R apart, applies the twiddles of its position k within
// the current sub-transform, does an R-point DFT in registers and writes the outputs Ns
// apart, ping-ponging between two buffers.  Radices 2, 3, 4, 5, 8 and the composite register
// codelets 6, 10, 12, 16 cover every 2*3*5-smooth length.  Conventions are FFTW's: sign -1 forward, +1 backward, both unnormalised.
//
// Twiddles come from a table tw[t] = exp(-2 pi i t / n) built on the host in extended
// precision and rounded once to the working type.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace clk {

template <typename T>
struct alignas(2 * sizeof(T)) cx {
    T re, im;
};

template <typename T>
__device__ __forceinline__ cx<T> mk(T r, T i) {
    cx<T> c;
    c.re = r;
    c.im = i;
    return c;
}
template <typename T>
__device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename T>
__device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename T>
__device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
__device__ __forceinline__ cx<T> cmulc(cx<T> a, cx<T> b) {  // a * conj(b)
    return mk(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im);
}
template <typename T>
__device__ __forceinline__ cx<T> scale(cx<T> a, T s) { return mk(a.re * s, a.im * s); }
// i * s * a for s = +-1
template <int S, typename T>
__device__ __forceinline__ cx<T> mul_is(cx<T> a) {
    return S > 0 ? mk(-a.im, a.re) : mk(a.im, -a.re);
}

// Decimal values of the DFT constants (exact mathematical constants rounded by the compiler).
#define CLK_SQRT1_2 0.70710678118654752440084436210484903928
#define CLK_SIN60 0.86602540378443864676372317075293618347      // sin(2 pi/3)
#define CLK_C1_5 0.30901699437494742410229341718281905886       // cos(2 pi/5)
#define CLK_C2_5 (-0.80901699437494742410229341718281905886)    // cos(4 pi/5)
#define CLK_S1_5 0.95105651629515357211643933337938214340       // sin(2 pi/5)
#define CLK_S2_5 0.58778525229247312916870595463907276860       // sin(4 pi/5)

// R-point DFTs in registers: v[k] <- sum_j v[j] exp(S * 2 pi i j k / R).
template <int S, typename T>
__device__ __forceinline__ void dft2(cx<T>* v) {
    cx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}

template <int S, typename T>
__device__ __forceinline__ void dft3(cx<T>* v) {
    const T h = T(0.5), s60 = T(CLK_SIN60);
    cx<T> t1 = v[1] + v[2];
    cx<T> t2 = v[0] - scale(t1, h);
    cx<T> t3 = mul_is<S>(scale(v[1] - v[2], s60));
    v[0] = v[0] + t1;
    v[1] = t2 + t3;
    v[2] = t2 - t3;
}

template <int S, typename T>
__device__ __forceinline__ void dft4(cx<T>* v) {
    cx<T> a = v[0] + v[2], b = v[0] - v[2];
    cx<T> c = v[1] + v[3], d = mul_is<S>(v[1] - v[3]);
    v[0] = a + c;
    v[2] = a - c;
    v[1] = b + d;
    v[3] = b - d;
}

template <int S, typename T>
__device__ __forceinline__ void dft5(cx<T>* v) {
    const T c1 = T(CLK_C1_5), c2 = T(CLK_C2_5), s1 = T(CLK_S1_5), s2 = T(CLK_S2_5);
    cx<T> a1 = v[1] + v[4], a2 = v[2] + v[3];
    cx<T> b1 = v[1] - v[4], b2 = v[2] - v[3];
    cx<T> x0 = v[0];
    cx<T> p1 = x0 + scale(a1, c1) + scale(a2, c2);
    cx<T> p2 = x0 + scale(a1, c2) + scale(a2, c1);
    cx<T> q1 = mul_is<S>(scale(b1, s1) + scale(b2, s2));
    cx<T> q2 = mul_is<S>(scale(b1, s2) - scale(b2, s1));
    v[0] = x0 + a1 + a2;
    v[1] = p1 + q1;
    v[4] = p1 - q1;
    v[2] = p2 + q2;
    v[3] = p2 - q2;
}

template <int S, typename T>
__device__ __forceinline__ void dft8(cx<T>* v) {
    cx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<S>(e);
    dft4<S>(o);
    const T r = T(CLK_SQRT1_2);
    // w8^k = exp(S i pi k / 4)
    cx<T> o1 = mk((o[1].re - S * o[1].im) * r, (o[1].im + S * o[1].re) * r);
    cx<T> o2 = mul_is<S>(o[2]);
    cx<T> o3 = mk((-o[3].re - S * o[3].im) * r, (-o[3].im + S * o[3].re) * r);
    v[0] = e[0] + o[0];
    v[4] = e[0] - o[0];
    v[1] = e[1] + o1;
    v[5] = e[1] - o1;
    v[2] = e[2] + o2;
    v[6] = e[2] - o2;
    v[3] = e[3] + o3;
    v[7] = e[3] - o3;
}

// 8-point DFT of (v[0..3], 0, 0, 0, 0): the zero half skipped (the zero-padded first stage of
// an aperiodic transform).
template <int S, typename T>
__device__ __forceinline__ void dft8_half_in(cx<T>* v) {
    const cx<T> e0 = v[0] + v[2], e2 = v[0] - v[2], is2 = mul_is<S>(v[2]);
    const cx<T> e1 = v[0] + is2, e3 = v[0] - is2;
    const cx<T> o0 = v[1] + v[3], o2 = v[1] - v[3], is3 = mul_is<S>(v[3]);
    const cx<T> p1 = v[1] + is3, p3 = v[1] - is3;
    const T r = T(CLK_SQRT1_2);
    const cx<T> o1 = mk((p1.re - S * p1.im) * r, (p1.im + S * p1.re) * r);
    const cx<T> o2w = mul_is<S>(o2);
    const cx<T> o3 = mk((-p3.re - S * p3.im) * r, (-p3.im + S * p3.re) * r);
    v[0] = e0 + o0;
    v[4] = e0 - o0;
    v[1] = e1 + o1;
    v[5] = e1 - o1;
    v[2] = e2 + o2w;
    v[6] = e2 - o2w;
    v[3] = e3 + o3;
    v[7] = e3 - o3;
}

// Outputs 0..3 of the 8-point DFT of v[0..7] (the kept half of an aperiodic result).
template <int S, typename T>
__device__ __forceinline__ void dft8_half_out(cx<T>* v) {
    cx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<S>(e);
    dft4<S>(o);
    const T r = T(CLK_SQRT1_2);
    const cx<T> o1 = mk((o[1].re - S * o[1].im) * r, (o[1].im + S * o[1].re) * r);
    const cx<T> o3 = mk((-o[3].re - S * o[3].im) * r, (-o[3].im + S * o[3].re) * r);
    v[0] = e[0] + o[0];
    v[1] = e[1] + o1;
    v[2] = e[2] + mul_is<S>(o[2]);
    v[3] = e[3] + o3;
}

template <int N>
struct WConst;
// Twiddle constants exp(2 pi i m / N) of the composite register codelets, evaluated to
// 40 digits from the Taylor series of cos and sin (generated once; values are exact
// mathematical constants, not taken from any library).
template <> struct WConst<6> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.5000000000000000000000000000000000000000;
            case 2: return -0.5000000000000000000000000000000000000000;
            case 3: return -1.0000000000000000000000000000000000000000;
            case 4: return -0.5000000000000000000000000000000000000000;
            case 5: return 0.5000000000000000000000000000000000000000;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.8660254037844386467637231707529361834714;
            case 2: return 0.8660254037844386467637231707529361834714;
            case 3: return 0.0000000000000000000000000000000000000000;
            case 4: return -0.8660254037844386467637231707529361834714;
            case 5: return -0.8660254037844386467637231707529361834714;
        }
        return 0.0;
    }
};
template <> struct WConst<10> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.8090169943749474241022934171828190588602;
            case 2: return 0.3090169943749474241022934171828190588602;
            case 3: return -0.3090169943749474241022934171828190588602;
            case 4: return -0.8090169943749474241022934171828190588602;
            case 5: return -1.0000000000000000000000000000000000000000;
            case 6: return -0.8090169943749474241022934171828190588602;
            case 7: return -0.3090169943749474241022934171828190588602;
            case 8: return 0.3090169943749474241022934171828190588602;
            case 9: return 0.8090169943749474241022934171828190588602;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.5877852522924731291687059546390727685977;
            case 2: return 0.9510565162951535721164393333793821434057;
            case 3: return 0.9510565162951535721164393333793821434057;
            case 4: return 0.5877852522924731291687059546390727685977;
            case 5: return 0.0000000000000000000000000000000000000000;
            case 6: return -0.5877852522924731291687059546390727685977;
            case 7: return -0.9510565162951535721164393333793821434057;
            case 8: return -0.9510565162951535721164393333793821434057;
            case 9: return -0.5877852522924731291687059546390727685977;
        }
        return 0.0;
    }
};
template <> struct WConst<12> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.8660254037844386467637231707529361834714;
            case 2: return 0.5000000000000000000000000000000000000000;
            case 3: return -0.0000000000000000000000000000000000000000;
            case 4: return -0.5000000000000000000000000000000000000000;
            case 5: return -0.8660254037844386467637231707529361834714;
            case 6: return -1.0000000000000000000000000000000000000000;
            case 7: return -0.8660254037844386467637231707529361834714;
            case 8: return -0.5000000000000000000000000000000000000000;
            case 9: return -0.0000000000000000000000000000000000000000;
            case 10: return 0.5000000000000000000000000000000000000000;
            case 11: return 0.8660254037844386467637231707529361834714;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.5000000000000000000000000000000000000000;
            case 2: return 0.8660254037844386467637231707529361834714;
            case 3: return 1.0000000000000000000000000000000000000000;
            case 4: return 0.8660254037844386467637231707529361834714;
            case 5: return 0.5000000000000000000000000000000000000000;
            case 6: return 0.0000000000000000000000000000000000000000;
            case 7: return -0.5000000000000000000000000000000000000000;
            case 8: return -0.8660254037844386467637231707529361834714;
            case 9: return -1.0000000000000000000000000000000000000000;
            case 10: return -0.8660254037844386467637231707529361834714;
            case 11: return -0.5000000000000000000000000000000000000000;
        }
        return 0.0;
    }
};
template <> struct WConst<16> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.9238795325112867561281831893967882868224;
            case 2: return 0.7071067811865475244008443621048490392848;
            case 3: return 0.3826834323650897717284599840303988667613;
            case 4: return -0.0000000000000000000000000000000000000000;
            case 5: return -0.3826834323650897717284599840303988667613;
            case 6: return -0.7071067811865475244008443621048490392848;
            case 7: return -0.9238795325112867561281831893967882868224;
            case 8: return -1.0000000000000000000000000000000000000000;
            case 9: return -0.9238795325112867561281831893967882868224;
            case 10: return -0.7071067811865475244008443621048490392848;
            case 11: return -0.3826834323650897717284599840303988667613;
            case 12: return -0.0000000000000000000000000000000000000000;
            case 13: return 0.3826834323650897717284599840303988667613;
            case 14: return 0.7071067811865475244008443621048490392848;
            case 15: return 0.9238795325112867561281831893967882868224;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.3826834323650897717284599840303988667613;
            case 2: return 0.7071067811865475244008443621048490392848;
            case 3: return 0.9238795325112867561281831893967882868224;
            case 4: return 1.0000000000000000000000000000000000000000;
            case 5: return 0.9238795325112867561281831893967882868224;
            case 6: return 0.7071067811865475244008443621048490392848;
            case 7: return 0.3826834323650897717284599840303988667613;
            case 8: return 0.0000000000000000000000000000000000000000;
            case 9: return -0.3826834323650897717284599840303988667613;
            case 10: return -0.7071067811865475244008443621048490392848;
            case 11: return -0.9238795325112867561281831893967882868224;
            case 12: return -1.0000000000000000000000000000000000000000;
            case 13: return -0.9238795325112867561281831893967882868224;
            case 14: return -0.7071067811865475244008443621048490392848;
            case 15: return -0.3826834323650897717284599840303988667613;
        }
        return 0.0;
    }
};

template <> struct WConst<9> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.7660444431189780352023926505554166739358;
            case 2: return 0.1736481776669303488517166267693147960004;
            case 3: return -0.5000000000000000000000000000000000000000;
            case 4: return -0.9396926207859083840541092773247314699362;
            case 5: return -0.9396926207859083840541092773247314699362;
            case 6: return -0.5000000000000000000000000000000000000000;
            case 7: return 0.1736481776669303488517166267693147960004;
            case 8: return 0.7660444431189780352023926505554166739358;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.6427876096865393263226434099072634329076;
            case 2: return 0.9848077530122080593667430245895230136706;
            case 3: return 0.8660254037844386467637231707529361834714;
            case 4: return 0.3420201433256687330440996146822595807631;
            case 5: return -0.3420201433256687330440996146822595807631;
            case 6: return -0.8660254037844386467637231707529361834714;
            case 7: return -0.9848077530122080593667430245895230136706;
            case 8: return -0.6427876096865393263226434099072634329076;
        }
        return 0.0;
    }
};
template <> struct WConst<15> {
    static __device__ __forceinline__ double c(int m) {
        switch (m) {
            case 0: return 1.0000000000000000000000000000000000000000;
            case 1: return 0.9135454576426008955021275719853171779408;
            case 2: return 0.6691306063588582138262733306867804735996;
            case 3: return 0.3090169943749474241022934171828190588602;
            case 4: return -0.1045284632676534713998341548024981190807;
            case 5: return -0.5000000000000000000000000000000000000000;
            case 6: return -0.8090169943749474241022934171828190588602;
            case 7: return -0.9781476007338056379285667478695995324597;
            case 8: return -0.9781476007338056379285667478695995324597;
            case 9: return -0.8090169943749474241022934171828190588602;
            case 10: return -0.5000000000000000000000000000000000000000;
            case 11: return -0.1045284632676534713998341548024981190807;
            case 12: return 0.3090169943749474241022934171828190588602;
            case 13: return 0.6691306063588582138262733306867804735996;
            case 14: return 0.9135454576426008955021275719853171779408;
        }
        return 0.0;
    }
    static __device__ __forceinline__ double s(int m) {
        switch (m) {
            case 0: return 0.0000000000000000000000000000000000000000;
            case 1: return 0.4067366430758002077539859903414976129231;
            case 2: return 0.7431448254773942350146970489742569771891;
            case 3: return 0.9510565162951535721164393333793821434057;
            case 4: return 0.9945218953682733369226919449805703815208;
            case 5: return 0.8660254037844386467637231707529361834714;
            case 6: return 0.5877852522924731291687059546390727685977;
            case 7: return 0.2079116908177593371017422844051251662166;
            case 8: return -0.2079116908177593371017422844051251662166;
            case 9: return -0.5877852522924731291687059546390727685977;
            case 10: return -0.8660254037844386467637231707529361834714;
            case 11: return -0.9945218953682733369226919449805703815208;
            case 12: return -0.9510565162951535721164393333793821434057;
            case 13: return -0.7431448254773942350146970489742569771891;
            case 14: return -0.4067366430758002077539859903414976129231;
        }
        return 0.0;
    }
};
template <int R, int S, typename T>
__device__ __forceinline__ void dft(cx<T>* v);

// Composite N = N1*N2 codelet in registers (decimation in time):
//   X[k1 + N1 k2] = sum_t W_N2^(t k2) [ W_N^(t k1) sum_j1 x[t + N2 j1] W_N1^(j1 k1) ].
template <int N1, int N2, int S, typename T>
__device__ __forceinline__ void dft_2f(cx<T>* v) {
    constexpr int N = N1 * N2;
    cx<T> y[N];
#pragma unroll
    for (int t = 0; t < N2; ++t) {
        cx<T> u[N1];
#pragma unroll
        for (int j = 0; j < N1; ++j) u[j] = v[t + N2 * j];
        dft<N1, S>(u);
#pragma unroll
        for (int k = 0; k < N1; ++k) {
            const int m = (t * k) % N;
            if (m == 0) {
                y[k * N2 + t] = u[k];
            } else {
                const cx<T> w = mk(T(WConst<N>::c(m)), T(S * WConst<N>::s(m)));
                y[k * N2 + t] = cmul(u[k], w);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < N1; ++k) {
        cx<T> w2[N2];
#pragma unroll
        for (int t = 0; t < N2; ++t) w2[t] = y[k * N2 + t];
        dft<N2, S>(w2);
#pragma unroll
        for (int q = 0; q < N2; ++q) v[k + N1 * q] = w2[q];
    }
}

template <int R, int S, typename T>
__device__ __forceinline__ void dft(cx<T>* v) {
    if constexpr (R == 1) return;  // a one-point DFT is the identity
    else if constexpr (R == 2) dft2<S>(v);
    else if constexpr (R == 3) dft3<S>(v);
    else if constexpr (R == 4) dft4<S>(v);
    else if constexpr (R == 5) dft5<S>(v);
    else if constexpr (R == 6) dft_2f<2, 3, S>(v);
    else if constexpr (R == 9) dft_2f<3, 3, S>(v);
    else if constexpr (R == 15) dft_2f<3, 5, S>(v);
    else if constexpr (R == 10) dft_2f<2, 5, S>(v);
    else if constexpr (R == 12) dft_2f<4, 3, S>(v);
    else if constexpr (R == 16) dft_2f<4, 4, S>(v);
    else dft8<S>(v);
}

// Exact quotient j / d for j, d < 2^16 from m = floor(2^32 / d) + 1; d = 1 wraps m to 0,
// which is taken to mean the identity.
__device__ __forceinline__ int fdiv(int j, unsigned m) { return m ? (int)__umulhi((unsigned)j, m) : j; }
__host__ __device__ inline unsigned fdiv_magic(int d) { return (unsigned)(0xFFFFFFFFu / (unsigned)d) + 1u; }

// Radix schedule of one axis.  Passed by value as a kernel parameter.
struct FftPlan {
    int n;
    int nst;
    int radix[16];
    unsigned ns_magic[16];  // fdiv_magic(product of the radices before stage s)
};

// One Stockham stage over `lines` lines in column layout.
template <int R, int S, typename T>
__device__ __forceinline__ void stage(const cx<T>* __restrict__ src, cx<T>* __restrict__ dst,
                                      const cx<T>* __restrict__ tw, int n, int ns, unsigned ns_m, int lines,
                                      unsigned lines_m, int ld) {
    const int nb = n / R;
    const int total = nb * lines;
    const int twstep = n / (ns * R);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        const int j = fdiv(b, lines_m);
        const int line = b - j * lines;
        const int k = j - fdiv(j, ns_m) * ns;
        cx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * ld + line];
        if (ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cx<T> w = tw[r * k * twstep];
                v[r] = S < 0 ? cmul(v[r], w) : cmulc(v[r], w);
            }
        }
        dft<R, S>(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(base + r * ns) * ld + line] = v[r];
    }
}

// Full transform of every line; returns the buffer (a or b) that holds the result.
// Must be called by every thread of the block; ends with a __syncthreads().
template <int S, typename T>
__device__ cx<T>* fft_lines(cx<T>* a, cx<T>* b, const cx<T>* __restrict__ tw, const FftPlan& p,
                            int lines, int ld) {
    int ns = 1;
    const unsigned lm = fdiv_magic(lines);
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s];
        const unsigned nm = p.ns_magic[s];
        switch (R) {
            case 2: stage<2, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 3: stage<3, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 4: stage<4, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 5: stage<5, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 6: stage<6, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 10: stage<10, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 12: stage<12, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            case 16: stage<16, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
            default: stage<8, S>(a, b, tw, p.n, ns, nm, lines, lm, ld); break;
        }
        __syncthreads();
        cx<T>* t = a;
        a = b;
        b = t;
        ns *= R;
    }
    return a;
}

}  // namespace clk

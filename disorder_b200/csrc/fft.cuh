// In-shared-memory mixed-radix Stockham FFT over a tile of L lines.
//
// A tile holds L lines of length N in shared memory with element (p, l) at
// buf[p * pitch + l] (line index fastest, pitch = L + 1 to spread banks).
// One stage of radix R reads R values spaced N/R apart, applies the twiddles
// exp(-2*pi*i*r*k/(Ns*R)), does an R-point DFT in registers and writes the
// results in Stockham (self-sorting) order, ping-ponging between two
// buffers. The algorithm is the mixed-radix Stockham formulation published
// by Govindaraju et al. ("High performance discrete Fourier transforms on
// graphics processors", SC 2008). Forward transforms use exp(-2*pi*i/N)
// (MATLAB's dftmtx convention); inverse transforms are formed by the caller
// as conj(FFT(conj(.))).
#pragma once
#include "common.cuh"

#define DIS_MAX_STAGES 12

struct FFTPlan {
  int n;
  int nst;
  int radix[DIS_MAX_STAGES];
};

// Host helper: factor n into radices 8,4,2,3,5,7,11,13 (largest power-of-two
// radices first). Returns false when another prime factor remains.
inline bool dis_make_fft_plan(int n, FFTPlan* p) {
  p->n = n;
  p->nst = 0;
  int m = n;
  const int rs[] = {8, 4, 2, 3, 5, 7, 11, 13};
  for (int r : rs) {
    while (m % r == 0) {
      if (p->nst >= DIS_MAX_STAGES) return false;
      p->radix[p->nst++] = r;
      m /= r;
    }
  }
  if (n == 1) {
    p->nst = 0;
    return true;
  }
  return m == 1;
}

// R-point forward DFTs on registers (exp(-2*pi*i*q*r/R)).
template <int R>
struct SmallDFT;

template <>
struct SmallDFT<2> {
  static DIS_D void run(float2* v, const float2*, int) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <>
struct SmallDFT<4> {
  static DIS_D void run(float2* v, const float2*, int) {
    float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, cmulmi(b1));  // a1 - i b1
    v[3] = csub(a1, cmulmi(b1));  // a1 + i b1
  }
};

template <>
struct SmallDFT<8> {
  static DIS_D void run(float2* v, const float2*, int) {
    const float h = 0.70710678118654752440f;  // cos(pi/4)
    // radix-2 split into even/odd 4-point DFTs
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    SmallDFT<4>::run(e, nullptr, 0);
    SmallDFT<4>::run(o, nullptr, 0);
    // twiddles exp(-2*pi*i*q/8) for q=0..3
    float2 t1 = make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));   // *(h - i h)
    float2 t2 = cmulmi(o[2]);                                                 // *(-i)
    float2 t3 = make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));  // *(-h - i h)
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  }
};

// Odd radices: pairwise symmetric evaluation. With a_r = v_r + v_{R-r} and
// b_r = v_r - v_{R-r}, X_q = v_0 + sum_r a_r cos(2 pi q r/R) - i sum_r b_r
// sin(2 pi q r/R) and X_{R-q} the same with +i. The cos/sin values come from
// the N-point twiddle table tw[m] = exp(-2*pi*i*m/N) (stride = N/R), so
// cos = tw.x and -sin = tw.y.
template <int R>
struct SmallDFT {
  static DIS_D void run(float2* v, const float2* tw, int stride) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
    float2 sum = v[0];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      a[r - 1] = cadd(v[r], v[R - r]);
      b[r - 1] = csub(v[r], v[R - r]);
      sum = cadd(sum, a[r - 1]);
    }
    float2 out[R];
    out[0] = sum;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      float2 A = v[0];
      float2 B = make_float2(0.f, 0.f);
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const int m = (q * r) % R;
        const float2 w = tw[m * stride];  // (cos, -sin) of 2 pi m / R
        A.x = fmaf(a[r - 1].x, w.x, A.x);
        A.y = fmaf(a[r - 1].y, w.x, A.y);
        B.x = fmaf(b[r - 1].x, w.y, B.x);  // B = sum b_r * (-sin)
        B.y = fmaf(b[r - 1].y, w.y, B.y);
      }
      // X_q = A + i*B (since -i*sin*b = i*(-sin)*b), X_{R-q} = A - i*B
      out[q] = cadd(A, cmuli(B));
      out[R - q] = csub(A, cmuli(B));
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
  }
};

template <int R>
DIS_D void fft_stage(const float2* __restrict__ src, float2* __restrict__ dst,
                     const float2* __restrict__ tw, int N, int L, int pitch, int Ns,
                     int tid, int nthr) {
  const int B = N / R;
  const int twStep = N / (Ns * R);
  const int total = L * B;
  for (int w = tid; w < total; w += nthr) {
    const int l = w % L;
    const int j = w / L;
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * B) * pitch + l];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[r * k * twStep]);
    }
    SmallDFT<R>::run(v, tw, N / R);
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(idxD + r * Ns) * pitch + l] = v[r];
  }
}

// Forward FFT of all L lines held in buffer a (using b as scratch).
// Returns the buffer that holds the result. Includes the trailing barrier.
DIS_D float2* fft_tile(float2* a, float2* b, const float2* tw, const FFTPlan& plan, int L,
                       int pitch, int tid, int nthr) {
  const int N = plan.n;
  int Ns = 1;
  for (int s = 0; s < plan.nst; ++s) {
    const int R = plan.radix[s];
    switch (R) {
      case 8: fft_stage<8>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 4: fft_stage<4>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 2: fft_stage<2>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 3: fft_stage<3>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 5: fft_stage<5>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 7: fft_stage<7>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 11: fft_stage<11>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      case 13: fft_stage<13>(a, b, tw, N, L, pitch, Ns, tid, nthr); break;
      default: break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// Twiddle table tw[m] = exp(-2*pi*i*m/N), m < N, evaluated in double
// precision and rounded to single; written to shared memory by the block.
DIS_D void load_twiddles(float2* tw, int N, int tid, int nthr) {
  for (int m = tid; m < N; m += nthr) {
    double s, c;
    sincospi(-2.0 * (double)m / (double)N, &s, &c);
    tw[m] = make_float2((float)c, (float)s);
  }
}

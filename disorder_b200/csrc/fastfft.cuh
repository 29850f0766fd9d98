// Register-resident line FFTs of compile-time length N = N1 * N2
// (N1, N2 <= 16), one line per group of TL = pow2ceil(max(N1,N2)) threads.
//
// Four-step factorisation (Bailey): with n = t + N2*m and k = k1 + N1*k2,
//   X[k] = sum_t W_N^{t k1} W_N2^{t k2} sum_m W_N1^{m k1} x[t + N2 m].
// Layout A: thread t < N2 holds a[m] = x[t + N2*m], m < N1 (space order).
// Layout B: thread k1 < N1 holds c[k2] = X[k1 + N1*k2], k2 < N2 (frequency).
// fwd(): A -> B; inv(): B -> A (unnormalised inverse DFT). Each does one
// exchange through a per-line shared-memory tile, synchronised with
// __syncwarp because a line never spans two warps (TL divides 32).
#pragma once
#include "common.cuh"

namespace ff {

template <int A, int B>
struct Max {
  static constexpr int v = A > B ? A : B;
};

constexpr int pow2ceil(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// ---------------------------------------------------------------- roots of unity
// exp(-2 pi i q / R) for the small DFTs, evaluated at compile time from the
// Taylor series of sin and cos about 0 (|angle| <= pi, 30 terms: converged
// to double precision) and rounded to single; the kernels read them from
// constant memory with compile-time offsets.
constexpr double kPi = 3.14159265358979323846;
constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int n = 1; n < 30; ++n) {
    t *= -x * x / ((2.0 * n) * (2.0 * n + 1));
    s += t;
  }
  return s;
}
constexpr double taylor_cos(double x) {
  double t = 1, s = 1;
  for (int n = 1; n < 30; ++n) {
    t *= -x * x / ((2.0 * n - 1) * (2.0 * n));
    s += t;
  }
  return s;
}
template <int R>
struct Roots {
  float c[R];  // cos(2 pi q / R)
  float s[R];  // -sin(2 pi q / R)
  constexpr Roots() : c(), s() {
    for (int q = 0; q < R; ++q) {
      const double ang = 2 * kPi * (2 * q > R ? q - R : q) / R;
      c[q] = (float)taylor_cos(ang);
      s[q] = (float)(-taylor_sin(ang));
    }
  }
};
template <int R>
__constant__ Roots<R> c_roots = Roots<R>();

template <int R>
DIS_D float2 root(int q) {  // W_R^q, q < R known at compile time after unrolling
  return make_float2(c_roots<R>.c[q], c_roots<R>.s[q]);
}

// ---------------------------------------------------------------- small DFTs
template <bool INV>
DIS_D float2 rot90(float2 a) {  // multiply by -i (forward) or +i (inverse)
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV>
struct DFT {
  // generic: direct evaluation with pairwise symmetry for odd R
  static DIS_D void run(float2* v, const float2* tw, int st) {
    float2 out[R];
    if constexpr (R % 2 == 1) {
      constexpr int H = (R - 1) / 2;
      float2 a[H], b[H];
      float2 s0 = v[0];
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        a[r - 1] = cadd(v[r], v[R - r]);
        b[r - 1] = csub(v[r], v[R - r]);
        s0 = cadd(s0, a[r - 1]);
      }
      out[0] = s0;
#pragma unroll
      for (int q = 1; q <= H; ++q) {
        float2 A = v[0], B = make_float2(0.f, 0.f);
#pragma unroll
        for (int r = 1; r <= H; ++r) {
          const float2 w = root<R>((q * r) % R);  // (cos, -sin)
          A = cfmas(a[r - 1], w.x, A);
          B = cfmas(b[r - 1], w.y, B);
        }
        // forward: X_q = A + i B, X_{R-q} = A - i B (B carries -sin)
        const float2 iB = make_float2(-B.y, B.x);
        out[q] = INV ? csub(A, iB) : cadd(A, iB);
        out[R - q] = INV ? cadd(A, iB) : csub(A, iB);
      }
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        float2 acc = v[0];
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = root<R>((q * r) % R);
          if (INV) w.y = -w.y;
          acc = cfma(v[r], w, acc);
        }
        out[q] = acc;
      }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
  }
};

template <bool INV>
struct DFT<1, INV> {
  static DIS_D void run(float2*, const float2*, int) {}
};

template <bool INV>
struct DFT<2, INV> {
  static DIS_D void run(float2* v, const float2*, int) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct DFT<4, INV> {
  static DIS_D void run(float2* v, const float2*, int) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 b0 = cadd(v[1], v[3]), b1 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  }
};

template <bool INV>
struct DFT<8, INV> {
  static DIS_D void run(float2* v, const float2*, int) {
    const float h = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    DFT<4, INV>::run(e, nullptr, 0);
    DFT<4, INV>::run(o, nullptr, 0);
    // o[q] *= W8^q (forward) or conj (inverse)
    const float s = INV ? 1.f : -1.f;
    const float2 t1 = make_float2(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));
    const float2 t2 = rot90<INV>(o[2]);
    const float2 t3 = make_float2(-h * (o[3].x + s * o[3].y), h * (s * o[3].x - o[3].y));
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

template <bool INV>
struct DFT<16, INV> {
  // 16 = 4 x 4 in registers: x[j + 4m] -> DFT4 over m -> twiddle W16^{j k1}
  // -> DFT4 over j -> X[k1 + 4 k2]
  static DIS_D void run(float2* v, const float2*, int) {
    const float c1 = 0.92387953251128675613f;  // cos(pi/8)
    const float s1 = 0.38268343236508977173f;  // sin(pi/8)
    const float h = 0.70710678118654752440f;
    float2 y[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float2 t[4] = {v[j], v[j + 4], v[j + 8], v[j + 12]};
      DFT<4, INV>::run(t, nullptr, 0);
#pragma unroll
      for (int k = 0; k < 4; ++k) y[j][k] = t[k];
    }
    // twiddles W16^{j*k} for j,k in 1..3 (forward: exp(-2 pi i jk/16))
    const float sg = INV ? 1.f : -1.f;
    auto tw = [&](float2 a, float c, float s) { return make_float2(a.x * c - sg * a.y * s, a.y * c + sg * a.x * s); };
    y[1][1] = tw(y[1][1], c1, s1);
    y[1][2] = tw(y[1][2], h, h);
    y[1][3] = tw(y[1][3], s1, c1);
    y[2][1] = tw(y[2][1], h, h);
    y[2][2] = rot90<INV>(y[2][2]);
    y[2][3] = tw(y[2][3], -h, h);
    y[3][1] = tw(y[3][1], s1, c1);
    y[3][2] = tw(y[3][2], -h, h);
    y[3][3] = tw(y[3][3], -c1, -s1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float2 t[4] = {y[0][k], y[1][k], y[2][k], y[3][k]};
      DFT<4, INV>::run(t, nullptr, 0);
#pragma unroll
      for (int q = 0; q < 4; ++q) v[k + 4 * q] = t[q];
    }
  }
};

// R = P*Q in registers (same four-step split as the line FFT):
// X[k1 + P k2] = sum_j W_R^{j k1} W_Q^{j k2} sum_m W_P^{m k1} x[j + Q m].
// W_R^{j k1} comes from root<R>(); the P- and Q-point DFTs use their own roots.
template <int P, int Q, bool INV>
struct DFT2D {
  static DIS_D void run(float2* v, const float2* tw, int st) {
    float2 y[Q][P];
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      float2 t[P];
#pragma unroll
      for (int m = 0; m < P; ++m) t[m] = v[j + Q * m];
      DFT<P, INV>::run(t, tw, st * Q);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        if (j == 0 || k1 == 0) {
          y[j][k1] = t[k1];
        } else {
          float2 w = root<P * Q>((j * k1) % (P * Q));
          if (INV) w.y = -w.y;
          y[j][k1] = cmul(t[k1], w);
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      float2 t[Q];
#pragma unroll
      for (int j = 0; j < Q; ++j) t[j] = y[j][k1];
      DFT<Q, INV>::run(t, tw, st * P);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = t[k2];
    }
  }
};

template <bool INV>
struct DFT<6, INV> : DFT2D<2, 3, INV> {};
template <bool INV>
struct DFT<10, INV> : DFT2D<2, 5, INV> {};
template <bool INV>
struct DFT<12, INV> : DFT2D<4, 3, INV> {};
template <bool INV>
struct DFT<14, INV> : DFT2D<2, 7, INV> {};
template <bool INV>
struct DFT<15, INV> : DFT2D<5, 3, INV> {};
template <bool INV>
struct DFT<9, INV> : DFT2D<3, 3, INV> {};

// ---------------------------------------------------------------- twiddles
// Shared-memory twiddles of a line FFT of length N = N1*N2 (SIZE float2):
//   [t*Q + k] = W_N^{t k}   (t, k < M = max(N1, N2))
// The forward step reads row t (its lane) at k = k1 and the inverse step row
// t at k = u, two entries per 16-byte load. The row pitch Q is twice an odd
// number, so 16 lanes reading the same column pair of their own rows hit the
// minimum two wavefronts. P is the (odd) pitch of the exchange tiles.
template <int N1, int N2>
struct Tw {
  static constexpr int M = N1 > N2 ? N1 : N2;
  static constexpr int Q0 = (M + 1) & ~1;
  static constexpr int Q = ((Q0 / 2) % 2 == 1) ? Q0 : Q0 + 2;
  static constexpr int SIZE = M * Q;
  static constexpr int P = (N2 % 2 == 0) ? N2 + 1 : N2 + 2;
};

// Fill the table above from the N-point table twg[m] = W_N^m (global memory).
template <int N1, int N2>
DIS_D void load_tw(float2* tws, const float2* __restrict__ twg, int tid, int nthr) {
  using T = Tw<N1, N2>;
  constexpr int N = N1 * N2;
  for (int e = tid; e < T::SIZE; e += nthr) {
    const int t = e / T::Q, k = e % T::Q;
    tws[e] = k < T::M ? twg[(t * k) % N] : make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------- line FFT
template <int N1_, int N2_>
struct Line {
  static constexpr int N1 = N1_;
  static constexpr int N2 = N2_;
  static constexpr int N = N1 * N2;
  static constexpr int TL = pow2ceil(Max<N1, N2>::v);  // threads per line
  static constexpr int EX = Tw<N1, N2>::P;             // exchange row pitch (odd: conflict-free)
  static constexpr int EXSZ = N1 * EX;                 // exchange tile per line (float2)
  static constexpr int TWS = Tw<N1, N2>::SIZE;         // shared twiddle table (float2)

  // A -> B. a: layout A (used when t < N2); c: layout B (valid when t < N1)
  static DIS_D void fwd(float2 (&a)[N1], float2 (&c)[N2], int t, float2* ex, const float2* tw) {
    using T = Tw<N1, N2>;
    static_assert(N1 % 2 == 0, "paired twiddle loads");
    if (t < N2) {
      DFT<N1, false>::run(a, nullptr, 1);
      const float4* tr = reinterpret_cast<const float4*>(tw + t * T::Q);
#pragma unroll
      for (int j = 0; j < N1 / 2; ++j) {
        const float4 w = tr[j];
        if (j > 0) a[2 * j] = cmul(a[2 * j], make_float2(w.x, w.y));
        a[2 * j + 1] = cmul(a[2 * j + 1], make_float2(w.z, w.w));
      }
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) ex[k1 * EX + t] = a[k1];
    }
    __syncwarp();
    if (t < N1) {
#pragma unroll
      for (int u = 0; u < N2; ++u) c[u] = ex[t * EX + u];
      DFT<N2, false>::run(c, nullptr, 1);
    }
    __syncwarp();
  }

  // B -> A, unnormalised inverse.
  static DIS_D void inv(float2 (&c)[N2], float2 (&a)[N1], int t, float2* ex, const float2* tw) {
    using T = Tw<N1, N2>;
    if (t < N1) {
      DFT<N2, true>::run(c, nullptr, 1);
      const float4* tr = reinterpret_cast<const float4*>(tw + t * T::Q);
#pragma unroll
      for (int j = 0; j < (N2 + 1) / 2; ++j) {
        const float4 w = tr[j];
        if (j > 0) c[2 * j] = cmulc(c[2 * j], make_float2(w.x, w.y));
        if (2 * j + 1 < N2) c[2 * j + 1] = cmulc(c[2 * j + 1], make_float2(w.z, w.w));
      }
#pragma unroll
      for (int u = 0; u < N2; ++u) ex[t * EX + u] = c[u];
    }
    __syncwarp();
    if (t < N2) {
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) a[k1] = ex[k1 * EX + t];
      DFT<N1, true>::run(a, nullptr, 1);
    }
    __syncwarp();
  }
};

}  // namespace ff

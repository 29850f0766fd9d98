// Tiles of lines for the shared-memory line kernels (passes.cu, shearlet.cu).
//
// A tile is L lines of an N0 x N1 x N2 volume (element (n0,n1,n2) at
// n0 + N0*(n1 + N1*n2)) along one axis. Axis-0 tiles are L consecutive
// contiguous lines; axis-1/2 tiles are L lines adjacent along axis 0, so that
// every row of the tile (one position along the axis) is a contiguous run in
// memory. In shared memory, element (p, l) (position p of line l) sits at
// buf[p * P + l] with an odd pitch P.
#pragma once
#include "common.cuh"

constexpr int kMaxL = 32;

struct LineTile {
  long long base[kMaxL];
  int coord[kMaxL][3];
  bool valid[kMaxL];
};

// Line enumeration of a tile for a pass along `axis` of an N0 x N1 x N2
// volume (element (n0,n1,n2) at n0 + N0*(n1 + N1*n2)). Axis-0 tiles are L
// consecutive contiguous lines; axis-1/2 tiles are L lines adjacent along
// axis 0 so that every row of the tile is a contiguous run in memory.
DIS_D void tile_lines(const int* N, int axis, int L, int tile, LineTile* t, int tid) {
  if (tid < L) {
    const int l = tid;
    long long base = 0;
    int c0 = 0, c1 = 0, c2 = 0;
    bool valid = true;
    if (axis == 0) {
      long long q = (long long)tile * L + l;
      valid = q < (long long)N[1] * N[2];
      c1 = (int)(q % N[1]);
      c2 = (int)(q / N[1]);
      base = q * N[0];
    } else {
      const int nt0 = (N[0] + L - 1) / L;
      const int other = tile / nt0;
      c0 = (tile % nt0) * L + l;
      valid = c0 < N[0];
      if (axis == 1) {
        c2 = other;
        base = c0 + (long long)c2 * N[0] * N[1];
      } else {
        c1 = other;
        base = c0 + (long long)c1 * N[0];
      }
    }
    // invalid lines (past the volume in a partial tile) get coordinate 0 so
    // that table rows looked up for them stay in range
    t->base[l] = valid ? base : 0;
    t->coord[l][0] = valid ? c0 : 0;
    t->coord[l][1] = valid ? c1 : 0;
    t->coord[l][2] = valid ? c2 : 0;
    t->valid[l] = valid;
  }
}

DIS_D long long axis_stride(const int* N, int axis) {
  return axis == 0 ? 1LL : (axis == 1 ? (long long)N[0] : (long long)N[0] * N[1]);
}

// Load a tile of lines into buf[p*P + l]; conj_in conjugates on the way.
DIS_D void load_tile(const float2* __restrict__ src, float2* buf, const LineTile& t, const int* N,
                     int axis, int n, int L, int P, bool conj_in, int tid, int nthr) {
  const long long st = axis_stride(N, axis);
  const int tot = n * L;
  if (axis == 0) {
    for (int e = tid; e < tot; e += nthr) {
      const int l = e / n, p = e - l * n;
      float2 v = t.valid[l] ? src[t.base[l] + p] : make_float2(0.f, 0.f);
      buf[p * P + l] = conj_in ? cconj(v) : v;
    }
  } else {
    for (int e = tid; e < tot; e += nthr) {
      const int p = e / L, l = e - p * L;
      float2 v = t.valid[l] ? src[t.base[l] + p * st] : make_float2(0.f, 0.f);
      buf[p * P + l] = conj_in ? cconj(v) : v;
    }
  }
}

template <class F>
DIS_D void for_tile(const LineTile& t, const int* N, int axis, int n, int L, int P, int tid, int nthr,
                    F&& f) {
  const long long st = axis_stride(N, axis);
  const int tot = n * L;
  if (axis == 0) {
    for (int e = tid; e < tot; e += nthr) {
      const int l = e / n, p = e - l * n;
      if (t.valid[l]) f(t.base[l] + p, p * P + l);
    }
  } else {
    for (int e = tid; e < tot; e += nthr) {
      const int p = e / L, l = e - p * L;
      if (t.valid[l]) f(t.base[l] + p * st, p * P + l);
    }
  }
}


// number of tiles of L lines for a pass along axis
inline size_t tiles_for(const int* N, int axis, int L) {
  if (axis == 0) return ((size_t)N[1] * N[2] + L - 1) / L;
  const size_t nt0 = (N[0] + L - 1) / L;
  return nt0 * (axis == 1 ? N[2] : N[1]);
}

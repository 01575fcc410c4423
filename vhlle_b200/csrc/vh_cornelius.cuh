// vh_cornelius.cuh -- Cornelius 4D iso-surface elements of one hypercube on
// the device (P. Huovinen and H. Petersen, Eur. Phys. J. A 48 (2012) 171,
// arXiv:1206.3371, as the reference's src/cornelius.cpp implements it).
//
// One warp handles one hypercube.  The 4-cube splits into 8 3-cubes
// (constant dimension i at j = 0, 1; cornelius.cpp:1733-1774), each 3-cube
// into 6 squares (:1436-1482).  A square gives 0-2 line elements from the
// cuts of its edges (:1083-1313), a 3-cube joins its lines into polygons
// (:1484-1578) and the 4-cube joins the polygons into polyhedra
// (:1776-1878).  Every polyhedron is one element; its centroid and normal
// come from the tetrahedra (line, polygon centroid, polyhedron mean) as in
// :761-935.  Every decision (cut tests, ambiguity rules, the line and
// polygon joining order, the 1e-10 point matching) and every floating-point
// operation follows the reference's order, so the elements are
// bit-identical to it.  Capacities: 96 lines, 64 polygons (8 per 3-cube),
// 10 elements, as the reference's arrays; a hypercube that would exceed
// them, or on which the reference stops (an odd number of cuts on a square,
// too few lines for a polygon), returns -1.  The squares go across the
// lanes, the 3-cubes across 8 lanes, and the joining into polyhedra and the
// reference-ordered sums run in one lane, all over shared memory (a thread
// per hypercube left ~2 warps per SM on a typical surface, each running the
// whole construction serially out of L2-resident local memory).
#pragma once

namespace vh {
namespace cn {

constexpr int kMaxLines = 96;
constexpr int kMaxPoly = 64;
constexpr int kMaxPolyPerCube = 8;
constexpr int kMaxElem = 10;
constexpr double kEps = 1e-10;

struct Line {
  double p[2][4];  // end points
  double o[4];     // a point outside the surface
  int start;       // which of p is the start point (flip_start_end swaps)
};

__device__ __forceinline__ const double* lstart(const Line& l) { return l.p[l.start]; }
__device__ __forceinline__ const double* lend(const Line& l) { return l.p[1 - l.start]; }

// Square::construct_lines with ends_of_edge and find_outside.  The square's
// constant dimensions are c0, c1 (values v0, v1), its corner values p[a][b]
// (a along x1, b along x2, x1 < x2).  Writes its 0-2 lines to out[0..n) and
// returns n; *amb_out = 1 when it is ambiguous, *err = 1 when the reference
// would stop (an odd number of cuts).
__device__ int square_lines(const double p[2][2], int c0, int c1, double v0, double v1, int x1,
                            int x2, const double* dx, double E0, Line* out, int* amb_out,
                            int* err) {
  *amb_out = 0;
  int above = 0;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
      if (p[i][j] >= E0) above++;
  if (above == 0 || above == 4) return 0;
  double cx[4], cy[4];
  int nc = 0;
  if ((p[0][0] - E0) * (p[1][0] - E0) < 0) {
    cx[nc] = (p[0][0] - E0) / (p[0][0] - p[1][0]) * dx[x1];
    cy[nc++] = 0;
  } else if (p[0][0] == E0 && p[1][0] < E0) {
    cx[nc] = 1e-9 * dx[x1];
    cy[nc++] = 0;
  } else if (p[1][0] == E0 && p[0][0] < E0) {
    cx[nc] = (1.0 - 1e-9) * dx[x1];
    cy[nc++] = 0;
  }
  if ((p[0][0] - E0) * (p[0][1] - E0) < 0) {
    cx[nc] = 0;
    cy[nc++] = (p[0][0] - E0) / (p[0][0] - p[0][1]) * dx[x2];
  } else if (p[0][0] == E0 && p[0][1] < E0) {
    cx[nc] = 0;
    cy[nc++] = 1e-9 * dx[x2];
  } else if (p[0][1] == E0 && p[0][0] < E0) {
    cx[nc] = 0;
    cy[nc++] = (1.0 - 1e-9) * dx[x2];
  }
  if ((p[1][0] - E0) * (p[1][1] - E0) < 0) {
    cx[nc] = dx[x1];
    cy[nc++] = (p[1][0] - E0) / (p[1][0] - p[1][1]) * dx[x2];
  } else if (p[1][0] == E0 && p[1][1] < E0) {
    cx[nc] = dx[x1];
    cy[nc++] = 1e-9 * dx[x2];
  } else if (p[1][1] == E0 && p[1][0] < E0) {
    cx[nc] = dx[x1];
    cy[nc++] = (1.0 - 1e-9) * dx[x2];
  }
  if ((p[0][1] - E0) * (p[1][1] - E0) < 0) {
    cx[nc] = (p[0][1] - E0) / (p[0][1] - p[1][1]) * dx[x1];
    cy[nc++] = dx[x2];
  } else if (p[0][1] == E0 && p[1][1] < E0) {
    cx[nc] = 1e-9 * dx[x1];
    cy[nc++] = dx[x2];
  } else if (p[1][1] == E0 && p[0][1] < E0) {
    cx[nc] = (1.0 - 1e-9) * dx[x1];
    cy[nc++] = dx[x2];
  }
  if (nc != 0 && nc != 2 && nc != 4) {
    *err = 1;
    return 0;
  }
  if (nc == 0) return 0;
  double ox[2], oy[2];
  int amb = 0;
  if (nc == 4) {
    amb = 1;
    double Emid = 0;
    Emid += 0.25 * p[0][0];
    Emid += 0.25 * p[0][1];
    Emid += 0.25 * p[1][0];
    Emid += 0.25 * p[1][1];
    if ((p[0][0] < E0 && Emid < E0) || (p[0][0] > E0 && Emid > E0)) {
      double t = cx[1];
      cx[1] = cx[2];
      cx[2] = t;
      t = cy[1];
      cy[1] = cy[2];
      cy[2] = t;
    }
    if ((Emid - E0) < 0) {
      ox[0] = ox[1] = 0.5 * dx[x1];
      oy[0] = oy[1] = 0.5 * dx[x2];
    } else if ((p[0][0] - E0) < 0) {
      ox[0] = 0;
      oy[0] = 0;
      ox[1] = dx[x1];
      oy[1] = dx[x2];
    } else {
      ox[0] = dx[x1];
      oy[0] = 0;
      ox[1] = 0;
      oy[1] = dx[x2];
    }
  } else {
    double sx = 0, sy = 0;
    int nout = 0;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++)
        if (p[i][j] < E0) {
          sx += i * dx[x1];
          sy += j * dx[x2];
          nout++;
        }
    ox[0] = sx;
    oy[0] = sy;
    ox[1] = oy[1] = 0;
    if (nout > 0) {
      ox[0] = ox[0] / (double)nout;
      oy[0] = oy[0] / (double)nout;
    }
  }
  for (int k = 0; k < nc / 2; k++) {
    Line& l = out[k];
#pragma unroll
    for (int e = 0; e < 2; e++) {
      l.p[e][x1] = cx[2 * k + e];
      l.p[e][x2] = cy[2 * k + e];
      l.p[e][c0] = v0;
      l.p[e][c1] = v1;
    }
    l.o[x1] = ox[k];
    l.o[x2] = oy[k];
    l.o[c0] = v0;
    l.o[c1] = v1;
    l.start = 0;
  }
  *amb_out = amb;
  return nc / 2;
}

// Polyhedron::tetravolume
__device__ __forceinline__ void tetra(const double* a, const double* b, const double* c,
                                      double* n) {
  const double bc01 = b[0] * c[1] - b[1] * c[0];
  const double bc02 = b[0] * c[2] - b[2] * c[0];
  const double bc03 = b[0] * c[3] - b[3] * c[0];
  const double bc12 = b[1] * c[2] - b[2] * c[1];
  const double bc13 = b[1] * c[3] - b[3] * c[1];
  const double bc23 = b[2] * c[3] - b[3] * c[2];
  n[0] = 1.0 / 6.0 * (a[1] * bc23 - a[2] * bc13 + a[3] * bc12);
  n[1] = -1.0 / 6.0 * (a[0] * bc23 - a[2] * bc03 + a[3] * bc02);
  n[2] = 1.0 / 6.0 * (a[0] * bc13 - a[1] * bc03 + a[3] * bc01);
  n[3] = -1.0 / 6.0 * (a[0] * bc12 - a[1] * bc02 + a[2] * bc01);
}

// Polyhedron::lines_equal
__device__ bool lines_equal(const Line& l1, const Line& l2) {
  const double *p11 = lstart(l1), *p12 = lend(l1), *p21 = lstart(l2);
  double d1 = 0, d2 = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    d1 += fabs(p11[i] - p21[i]);
    d2 += fabs(p12[i] - p21[i]);
    if (d1 > kEps && d2 > kEps) return false;
  }
  return true;
}

}  // namespace cn

// ---------------------------------------------------------------------
// The warp's part: 48 square instances (8 3-cubes x 6 squares) across the
// lanes, each 3-cube's polygons in one of 8 lanes, the joining into
// polyhedra in lane 0, the tetrahedra of the centroid and normal sums across
// the lanes.
namespace cnw {

using cn::kEps;
using cn::kMaxElem;
using cn::Line;
using cn::lend;
using cn::lstart;

struct Poly {
  unsigned char li[12];  // line ids: 2 * square instance + line
  int n;
  double cen[4];
};

struct WarpWork {
  Line L[96];  // lines of square instance t at 2t, 2t + 1
  unsigned char sqn[48], sqamb[48];
  Poly P[8][8];  // polygons of each 3-cube
  int np[8], nl[8], camb[8];
  double hc[16];
  int err;
  // the elements as tetrahedra (one per polygon line), in the order of the
  // reference's sums: element e owns tetrahedra es[e] .. es[e+1]-1
  unsigned char tp[96], tl[96];  // polygon code (8 * 3-cube + polygon), line id
  int es[kMaxElem + 1], nel;
  double term[96][5];  // per-tetrahedron terms of the current sum
};

// Square instance t = 6 c + s: 3-cube c (constant dimension c / 2 at corner
// bit c % 2), square s (its constant dimension the (s / 2)-th free dimension
// of the 3-cube, at bit s % 2) -- the order Cube::split_to_squares and
// Hypercube::split_to_cubes produce (src/cornelius.cpp:1436-1482,1733-1774).
__device__ __forceinline__ void square_instance(WarpWork& w, int t, const double* dx, double E0) {
  const int c = t / 6, s = t % 6, ci = c >> 1, jc = c & 1, j = s & 1;
  int fr[3], k = 0;
  for (int d = 0; d < 4; d++)
    if (d != ci) fr[k++] = d;
  const int i = fr[s >> 1];
  int x1 = -1, x2 = -1;
  for (int d = 0; d < 4; d++)
    if (d != ci && d != i) {
      if (x1 < 0)
        x1 = d;
      else
        x2 = d;
    }
  double sq[2][2];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++)
      sq[a][b] = w.hc[(jc << (3 - ci)) | (j << (3 - i)) | (a << (3 - x1)) | (b << (3 - x2))];
  int amb = 0, err = 0;
  const int n = cn::square_lines(sq, ci, i, jc * dx[ci], j * dx[i], x1, x2, dx, E0, &w.L[2 * t],
                                 &amb, &err);
  w.sqn[t] = (unsigned char)n;
  w.sqamb[t] = (unsigned char)amb;
  if (err) atomicOr(&w.err, 1);
}

// Polygon::add_line (src/cornelius.cpp:404-438)
__device__ bool add_line(WarpWork& w, Poly& pg, int li, bool donotcheck) {
  if (donotcheck || pg.n == 0) {
    pg.li[pg.n++] = (unsigned char)li;
    return true;
  }
  Line& l = w.L[li];
  const double *p1 = lstart(l), *p2 = lend(l), *p3 = lend(w.L[pg.li[pg.n - 1]]);
  double d1 = 0, d2 = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    d1 += fabs(p1[j] - p3[j]);
    d2 += fabs(p2[j] - p3[j]);
  }
  if (d1 < kEps || d2 < kEps) {
    if (d2 < kEps) l.start = 1 - l.start;
    pg.li[pg.n++] = (unsigned char)li;
    return true;
  }
  return false;
}

// Polygon::calculate_centroid (src/cornelius.cpp:440-516)
__device__ void poly_centroid(const WarpWork& w, Poly& pg, int cdim) {
  int x[3], k = 0;
  for (int d = 0; d < 4; d++)
    if (d != cdim) x[k++] = d;
  const int x1 = x[0], x2 = x[1], x3 = x[2];
  double mean[4] = {0, 0, 0, 0};
  for (int i = 0; i < pg.n; i++) {
    const Line& l = w.L[pg.li[i]];
    const double *p1 = lstart(l), *p2 = lend(l);
#pragma unroll
    for (int j = 0; j < 4; j++) mean[j] += p1[j] + p2[j];
  }
#pragma unroll
  for (int j = 0; j < 4; j++) mean[j] = mean[j] / (double)(2.0 * pg.n);
  if (pg.n == 3) {
#pragma unroll
    for (int j = 0; j < 4; j++) pg.cen[j] = mean[j];
    return;
  }
  double up[4] = {0, 0, 0, 0}, down = 0, a[4], b[4];
  for (int i = 0; i < pg.n; i++) {
    const Line& l = w.L[pg.li[i]];
    const double *p1 = lstart(l), *p2 = lend(l);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      a[j] = p1[j] - mean[j];
      b[j] = p2[j] - mean[j];
    }
    const double c1 = a[x2] * b[x3] - a[x3] * b[x2];
    const double c2 = a[x1] * b[x3] - a[x3] * b[x1];
    const double c3 = a[x2] * b[x1] - a[x1] * b[x2];
    const double A = 0.5 * sqrt(c1 * c1 + c2 * c2 + c3 * c3);
#pragma unroll
    for (int j = 0; j < 4; j++) up[j] += (p1[j] + p2[j] + mean[j]) / 3.0 * A;
    down += A;
  }
#pragma unroll
  for (int j = 0; j < 4; j++) pg.cen[j] = up[j] / down;
}

// Cube::construct_polygons + check_ambiguous for 3-cube c
// (src/cornelius.cpp:1484-1595), then its polygons' centroids.
__device__ void cube_polygons(WarpWork& w, int c) {
  unsigned char ids[12];
  int nl = 0, namb = 0;
  for (int s = 0; s < 6; s++) {
    const int t = 6 * c + s;
    namb += w.sqamb[t];
    for (int j = 0; j < w.sqn[t]; j++) ids[nl++] = (unsigned char)(2 * t + j);
  }
  w.nl[c] = nl;
  w.np[c] = 0;
  w.camb[c] = 0;
  if (nl == 0) return;
  int amb = namb;
  if (amb == 0 && nl == 6) amb = 1;
  w.camb[c] = amb;
  int np = 0;
  if (amb > 0) {
    unsigned unused = (1u << nl) - 1u;
    int used = 0;
    do {
      if (nl - used < 3 || np >= cn::kMaxPolyPerCube) {
        atomicOr(&w.err, 4);
        return;
      }
      Poly& pg = w.P[c][np];
      pg.n = 0;
      for (int i = 0; i < nl; i++) {
        if (((unused >> i) & 1u) && pg.n < 12) {
          if (add_line(w, pg, ids[i], false)) {
            unused &= ~(1u << i);
            used++;
            i = 0;
          }
        }
      }
      np++;
    } while (used < nl);
  } else {
    Poly& pg = w.P[c][0];
    pg.n = 0;
    for (int i = 0; i < nl; i++) add_line(w, pg, ids[i], true);
    np = 1;
  }
  w.np[c] = np;
  for (int q = 0; q < np; q++) poly_centroid(w, w.P[c][q], c >> 1);
}

// Hypercube::check_ambiguous + construct_polyhedrons (src/cornelius.cpp:
// 1776-1878), one lane: fills the tetrahedron list and w.nel (-1 where the
// reference stops).
__device__ void assemble(WarpWork& w, double E0) {
  int namb = 0, nlines = 0;
  unsigned char fl[64];  // polygons in the reference's order: 3-cube, then polygon
  int nf = 0;
  for (int c = 0; c < 8; c++) {
    if (w.camb[c]) namb++;
    nlines += w.nl[c];
    for (int q = 0; q < w.np[c]; q++) fl[nf++] = (unsigned char)(8 * c + q);
  }
  int amb = namb;
  if (amb == 0) {
    int pts = 0;
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (w.hc[k] < E0) pts++;
    if (pts > 8) pts = 16 - pts;
    if (nlines == 24 && pts == 2) amb++;
  }
  unsigned char ph[kMaxElem][64];
  int nph[kMaxElem], nel = 0;
  if (amb > 0) {
    unsigned long long unused = nf >= 64 ? ~0ull : ((1ull << nf) - 1);
    int used = 0;
    do {
      if (nel >= kMaxElem) {
        w.nel = -1;
        return;
      }
      nph[nel] = 0;
      for (int i = 0; i < nf; i++) {
        if (!((unused >> i) & 1)) continue;
        bool add = nph[nel] == 0;
        if (!add) {
          const Poly& p = w.P[fl[i] >> 3][fl[i] & 7];
          for (int q = 0; q < nph[nel] && !add; q++) {
            const Poly& pq = w.P[ph[nel][q] >> 3][ph[nel][q] & 7];
            for (int j = 0; j < p.n && !add; j++)
              for (int k = 0; k < pq.n && !add; k++)
                if (cn::lines_equal(w.L[p.li[j]], w.L[pq.li[k]])) add = true;
          }
        }
        if (add) {
          ph[nel][nph[nel]++] = fl[i];
          unused &= ~(1ull << i);
          used++;
          i = 0;
        }
      }
      nel++;
    } while (used < nf);
  } else {
    nph[0] = 0;
    for (int i = 0; i < nf; i++) ph[0][nph[0]++] = fl[i];
    nel = 1;
  }
  int nt = 0;
  for (int e = 0; e < nel; e++) {
    w.es[e] = nt;
    for (int q = 0; q < nph[e]; q++) {
      const Poly& pg = w.P[ph[e][q] >> 3][ph[e][q] & 7];
      for (int j = 0; j < pg.n; j++) {
        w.tp[nt] = ph[e][q];
        w.tl[nt] = pg.li[j];
        nt++;
      }
    }
  }
  w.es[nel] = nt;
  w.nel = nel;
}

// Polyhedron::calculate_centroid and calculate_normal (src/cornelius.cpp:
// 790-935) of element e, all lanes: each lane forms the terms of its
// tetrahedra, then every lane adds them in the reference's order (the same
// uniform sums in every lane).  Lane 0 writes geo[e][8].
__device__ void element(WarpWork& w, int e, double* geo) {
  const int lane = threadIdx.x & 31, t0 = w.es[e], t1 = w.es[e + 1];
  double mean[4] = {0, 0, 0, 0};
  for (int t = t0; t < t1; t++) {
    const Line& l = w.L[w.tl[t]];
    const double *p1 = lstart(l), *p2 = lend(l);
#pragma unroll
    for (int k = 0; k < 4; k++) mean[k] += p1[k] + p2[k];
  }
#pragma unroll
  for (int k = 0; k < 4; k++) mean[k] = mean[k] / (double)(2.0 * (t1 - t0));
  double a[4], b[4], c[4], n[4];
  for (int t = t0 + lane; t < t1; t += 32) {
    const Line& l = w.L[w.tl[t]];
    const Poly& pg = w.P[w.tp[t] >> 3][w.tp[t] & 7];
    const double *p1 = lstart(l), *p2 = lend(l);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      a[k] = p1[k] - mean[k];
      b[k] = p2[k] - mean[k];
      c[k] = pg.cen[k] - mean[k];
    }
    cn::tetra(a, b, c, n);
    double V = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) V += n[k] * n[k];
    V = sqrt(V);
#pragma unroll
    for (int k = 0; k < 4; k++) w.term[t][k] = (p1[k] + p2[k] + pg.cen[k] + mean[k]) / 4.0 * V;
    w.term[t][4] = V;
  }
  __syncwarp();
  double up[4] = {0, 0, 0, 0}, down = 0;
  for (int t = t0; t < t1; t++) {
#pragma unroll
    for (int k = 0; k < 4; k++) up[k] += w.term[t][k];
    down += w.term[t][4];
  }
  double C[4];
#pragma unroll
  for (int k = 0; k < 4; k++) C[k] = up[k] / down;
  __syncwarp();
  for (int t = t0 + lane; t < t1; t += 32) {
    const Line& l = w.L[w.tl[t]];
    const Poly& pg = w.P[w.tp[t] >> 3][w.tp[t] & 7];
    const double *p1 = lstart(l), *p2 = lend(l);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      a[k] = p1[k] - C[k];
      b[k] = p2[k] - C[k];
      c[k] = pg.cen[k] - C[k];
    }
    cn::tetra(a, b, c, n);
    double dot = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) dot += (l.o[k] - C[k]) * n[k];
    if (dot < 0) {
#pragma unroll
      for (int k = 0; k < 4; k++) n[k] = -n[k];
    }
#pragma unroll
    for (int k = 0; k < 4; k++) w.term[t][k] = n[k];
  }
  __syncwarp();
  double Nn[4] = {0, 0, 0, 0};
  for (int t = t0; t < t1; t++) {
#pragma unroll
    for (int k = 0; k < 4; k++) Nn[k] += w.term[t][k];
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      geo[e * 8 + k] = C[k];
      geo[e * 8 + 4 + k] = Nn[k];
    }
  }
  __syncwarp();
}

// The whole hypercube by the calling warp (every lane calls it, after the
// caller has put the 16 corner values into w.hc and synchronised the warp).
// Every lane gets the element count (-1 where the reference stops); lane 0
// has written the elements to geo.
__device__ int find_surface_warp(WarpWork& w, const double* dx, double E0, double* geo) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) w.err = 0;
  __syncwarp();
  // Cornelius::find_surface_4d: no elements unless the iso-value straddles
  // the corners (src/cornelius.cpp:2254-2268)
  int above = 0;
#pragma unroll
  for (int k = 0; k < 16; k++)
    if (w.hc[k] >= E0) above++;
  if (above == 0 || above == 16) return 0;  // uniform across the warp
  for (int t = lane; t < 48; t += 32) square_instance(w, t, dx, E0);
  __syncwarp();
  if (lane < 8) cube_polygons(w, lane);
  __syncwarp();
  if (lane == 0) {
    if (w.err)
      w.nel = -1;
    else
      assemble(w, E0);
  }
  __syncwarp();
  const int nel = w.nel;
  for (int e = 0; e < nel; e++) element(w, e, geo);
  return nel;
}

}  // namespace cnw
}  // namespace vh

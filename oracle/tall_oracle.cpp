// tall_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle), never part of the product.
//
// A float64 assembly of the restricted tall-cell pressure system at any size,
// the same system oracle/tall.py assembles with per-face Python loops (which
// only reach small grids).  It restates, paths relative to the
// peter-suggate/fluid tree:
//  * packed tall-cell layout          lib/core/tall-cell-grid.ts:171-190, 398-409
//    (sample 0 = the tall cell's bottom subcell, row 0; sample 1 = its top
//    subcell, row base - 1; sample j >= 2 = band row base + j - 2)
//  * linear tall-cell interpolation   docs/papers/tallCells.txt:155-161 (Eq. 5)
//  * face-row operator A = G^T W G    lib/methods/adaptive-mass/sparse-atlas-composite-projection.ts:381-620
//  * ghost-fluid theta                lib/core/cm12-numerics.ts:37-45 (epsilon 1e-12)
// Every face of the equivalent dense MAC grid with a liquid side adds
// (1/theta) g g^T, g = (samples representing the liquid side(s)) with weights,
// the liquid side's weights positive and the other side's negative; a dense
// cell in a tall segment is represented by its column's two tall samples
// weighted (1 - t, t), t = y / (base - 1); a band cell by its sample; rows
// above the band are air with phi = 0.5.  The right-hand side is
// b = T^T (-div u) over liquid dense cells, u interpolated the same way.
//
// Rows are assembled per column, in parallel: the column's vertical faces and
// the lateral faces to its four neighbours, kept only for the column's own rows
// (each lateral face is visited once from each side).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Tall {
  int nx, ny, nz, band, P;
  const int* bases;   // [nz][nx]
  const float* vof;   // [nz][P][nx]
  long idx(int x, int j, int z) const { return x + long(nx) * (j + long(P) * z); }
  int base(int x, int z) const { return bases[x + nx * z]; }
  // (liquid, phi) of dense cell (x, y, z); phi = 0.5 - vof of its sample
  bool cell(int x, int y, int z, double& phi) const {
    const int b = base(x, z);
    double f;
    if (y < b) {
      f = vof[idx(x, 0, z)];
    } else if (y < b + band) {
      f = vof[idx(x, y - b + 2, z)];
    } else {
      phi = 0.5;
      return false;
    }
    phi = 0.5 - f;
    return f > 0.5;
  }
  // representation of dense cell (x, y, z): up to two (sample, weight)
  int rep(int x, int y, int z, long* k, double* w) const {
    const int b = base(x, z);
    if (y < b) {
      const double t = double(y) / double(b - 1);
      k[0] = idx(x, 0, z);
      w[0] = 1.0 - t;
      k[1] = idx(x, 1, z);
      w[1] = t;
      return 2;
    }
    if (y < b + band) {
      k[0] = idx(x, y - b + 2, z);
      w[0] = 1.0;
      return 1;
    }
    return 0;
  }
};

double ghost_theta(double liquid_phi, double air_phi) {
  const double a = std::fabs(liquid_phi);
  return std::min(1.0, std::max(0.05, a / std::max(a + std::fabs(air_phi), 1e-12)));
}

}  // namespace

extern "C" {

// Assembles the tall-cell operator (CSR over all n = nx * P * nz samples,
// column-sorted rows, duplicates summed) and b = T^T (-div u).  indptr has
// n + 1 entries; indices / data are filled up to *nnz when they are non-null
// and cap >= the count (call once with null arrays to learn nnz).  Returns 0.
int orc_tall_assemble(int nx, int ny, int nz, int band, const int* bases, const float* vof, const float* u,
                      const float* v, const float* w, long* indptr, int* indices, double* data, long cap, long* nnz,
                      double* b) {
  Tall T{nx, ny, nz, band, band + 2, bases, vof};
  const int P = T.P;
  if (P > 64) return 1;
  const long n = long(nx) * P * nz, ncol = long(nx) * nz;
  // per column: sorted, summed rows (col, val) kept until the CSR is written
  std::vector<std::vector<std::pair<long, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 16)
  for (long c = 0; c < ncol; ++c) {
    const int x = int(c % nx), z = int(c / nx);
    // this column's rows (sample j of the column), entries unsorted until the end
    std::vector<long> cols[64];
    std::vector<double> vals[64];
    // one dense face's (1/theta) g g^T, kept for the rows of column c
    auto add_face = [&](int x0, int y0, int z0, int x1, int y1, int z1) {
      double pi, pj;
      const bool li = T.cell(x0, y0, z0, pi), lj = T.cell(x1, y1, z1, pj);
      if (!li && !lj) return;
      const double th = (li && lj) ? 1.0 : (li ? ghost_theta(pi, pj) : ghost_theta(pj, pi));
      long k[4];
      double wv[4];
      int m = 0;
      if (li) {
        long kk[2];
        double ww[2];
        const int q = T.rep(x0, y0, z0, kk, ww);
        for (int e = 0; e < q; ++e) { k[m] = kk[e]; wv[m++] = ww[e]; }
      }
      if (lj) {
        long kk[2];
        double ww[2];
        const int q = T.rep(x1, y1, z1, kk, ww);
        for (int e = 0; e < q; ++e) {
          int f = -1;
          for (int g = 0; g < m; ++g)
            if (k[g] == kk[e]) f = g;
          if (f >= 0) {
            wv[f] -= ww[e];
          } else {
            k[m] = kk[e];
            wv[m++] = -ww[e];
          }
        }
      }
      for (int a = 0; a < m; ++a) {
        if (wv[a] == 0.0) continue;
        // keep only rows of this column
        const long r = k[a];
        const long rx = r % nx, rz = r / (long(nx) * P), rj = (r / nx) % P;
        if (rx != x || rz != z) continue;
        for (int bb = 0; bb < m; ++bb) {
          if (wv[bb] == 0.0) continue;
          cols[rj].push_back(k[bb]);
          vals[rj].push_back(wv[a] * wv[bb] / th);
        }
      }
    };
    for (int y = 0; y < ny; ++y) {
      if (y + 1 < ny) add_face(x, y, z, x, y + 1, z);
      if (x + 1 < nx) add_face(x, y, z, x + 1, y, z);
      if (x > 0) add_face(x - 1, y, z, x, y, z);
      if (z + 1 < nz) add_face(x, y, z, x, y, z + 1);
      if (z > 0) add_face(x, y, z - 1, x, y, z);
    }
    for (int j = 0; j < P; ++j) {
      std::vector<std::pair<long, double>>& out = rows[T.idx(x, j, z)];
      std::vector<std::pair<long, double>> e(cols[j].size());
      for (size_t q = 0; q < e.size(); ++q) e[q] = {cols[j][q], vals[j][q]};
      std::sort(e.begin(), e.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      for (size_t q = 0; q < e.size();) {
        size_t r = q;
        double s = 0.0;
        while (r < e.size() && e[r].first == e[q].first) s += e[r++].second;
        out.push_back({e[q].first, s});
        q = r;
      }
    }
  }
  long total = 0;
  for (long r = 0; r < n; ++r) {
    indptr[r] = total;
    total += long(rows[r].size());
  }
  indptr[n] = total;
  *nnz = total;
  if (indices && data && cap >= total) {
#pragma omp parallel for schedule(static)
    for (long r = 0; r < n; ++r) {
      long o = indptr[r];
      for (const auto& e : rows[r]) {
        indices[o] = int(e.first);
        data[o++] = e.second;
      }
    }
  }
  // b = T^T (-div u) over liquid dense cells; a cell's faces are its own
  // representation's packed +faces and its negative neighbours' +faces
  if (b) {
    std::fill(b, b + n, 0.0);
    auto facev = [&](const float* a, int x, int y, int z) {
      long k[2];
      double wv[2];
      const int q = T.rep(x, y, z, k, wv);
      double s = 0.0;
      for (int e = 0; e < q; ++e) s += wv[e] * double(a[k[e]]);
      return s;
    };
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = 0; c < ncol; ++c) {
      const int x = int(c % nx), z = int(c / nx);
      for (int y = 0; y < ny; ++y) {
        double phi;
        if (!T.cell(x, y, z, phi)) continue;
        const double du = facev(u, x, y, z) - (x > 0 ? facev(u, x - 1, y, z) : 0.0);
        const double dv = facev(v, x, y, z) - (y > 0 ? facev(v, x, y - 1, z) : 0.0);
        const double dw = facev(w, x, y, z) - (z > 0 ? facev(w, x, y, z - 1) : 0.0);
        const double d = -((du + dw) + dv);
        long k[2];
        double wv[2];
        const int q = T.rep(x, y, z, k, wv);
        for (int e = 0; e < q; ++e) b[k[e]] += wv[e] * d;   // rows of column c only
      }
    }
  }
  return 0;
}

}  // extern "C"

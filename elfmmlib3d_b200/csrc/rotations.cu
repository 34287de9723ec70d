// rotations.cu -- translations factored as rotation, shift along z, rotation
// back: host construction of the factored operators and the device kernel.
//
// The rotation blocks are obtained by least-squares fits of the harmonic
// basis of one degree at fixed sample points on the unit sphere: the
// coefficients of a field in the rotated frame are those that reproduce the
// field's values at the sample points, mapped back through the rotation.
// This uses only the evaluation routines of harmonics.cuh (the same
// conventions as the dense operators, conjugate symmetry of real fields
// included), and check_factored_ops compares the product with the dense
// operator of every group.
#include <algorithm>
#include <cmath>
#include <random>
#include <thread>
#include <type_traits>
#include <cstdlib>
#include <cstring>
#include "common.cuh"
#include "harmonics.cuh"
#include "fmm.h"
#include "rotations.h"

namespace efmm {

namespace {

// offset (elements) of degree block n in a rotation part: sum_{j<n} (2j+2)^2
EFMM_HD long long rot_block_off(int n) { return (long long)2 * n * (n + 1) * (2 * n + 1) / 3; }
EFMM_HD long long rot_size(int p) { return rot_block_off(p + 1); }
// offset of order block m in a shift part: sum_{m'<m} (2(p-m'+1))^2
EFMM_HD long long sq_sum(long long x) { return x * (x + 1) * (2 * x + 1) / 6; }
EFMM_HD long long z_block_off(int p, int m) { return 4 * (sq_sum(p + 1) - sq_sum(p + 1 - m)); }
EFMM_HD long long z_size(int p) { return z_block_off(p, p + 1); }

// Value of the field of storage slot s (= 2m + part) of degree n at a point,
// from a harmonics table: multipole basis (irregular T, coefficient of T) or
// local basis (conjugated regular Y).
inline double slot_value(int basis, const cplx* tab, int n, int s) {
  const int m = s >> 1, part = s & 1;
  const double w = m == 0 ? 1.0 : 2.0;
  const cplx v = tab[cidx(n, m)];
  if (basis == 0) return part == 0 ? w * v.re : -w * v.im;
  return part == 0 ? w * v.re : w * v.im;
}

struct Fitter {
  int p = 0, K = 0;
  std::vector<double> pts;             // K x 3
  std::vector<std::vector<double>> pinv[2];  // [basis][n]: (2n+1) x K over active slots

  void init(int pmax) {
    p = pmax;
    K = 2 * (2 * p + 2) + 16;
    pts.resize(3 * (size_t)K);
    const double ga = M_PI * (3.0 - std::sqrt(5.0));
    for (int k = 0; k < K; k++) {
      double z = 1.0 - (2.0 * k + 1.0) / K, r = std::sqrt(std::max(0.0, 1.0 - z * z)), ph = ga * k;
      pts[3 * k] = r * std::cos(ph);
      pts[3 * k + 1] = r * std::sin(ph);
      pts[3 * k + 2] = z;
    }
    std::vector<cplx> tab(ncoef(p));
    std::vector<std::vector<cplx>> T(K), Y(K);
    for (int k = 0; k < K; k++) {
      T[k].resize(ncoef(p));
      Y[k].resize(ncoef(p));
      irregular_harmonics(p, pts[3 * k], pts[3 * k + 1], pts[3 * k + 2], T[k].data());
      regular_harmonics(p, pts[3 * k], pts[3 * k + 1], pts[3 * k + 2], Y[k].data());
    }
    for (int basis = 0; basis < 2; basis++) {
      pinv[basis].resize(p + 1);
      for (int n = 0; n <= p; n++) {
        const int b = 2 * n + 1;  // active slots: 0, then 2..2n+1
        // B (K x b), column-scaled, thin QR by modified Gram-Schmidt (twice)
        std::vector<double> Q((size_t)K * b), R((size_t)b * b, 0.0), sc(b);
        for (int j = 0; j < b; j++) {
          const int s = j == 0 ? 0 : j + 1;
          double nrm = 0;
          for (int k = 0; k < K; k++) {
            double v = slot_value(basis, basis == 0 ? T[k].data() : Y[k].data(), n, s);
            Q[(size_t)k * b + j] = v;
            nrm += v * v;
          }
          sc[j] = nrm > 0 ? 1.0 / std::sqrt(nrm) : 1.0;
          for (int k = 0; k < K; k++) Q[(size_t)k * b + j] *= sc[j];
        }
        for (int j = 0; j < b; j++) {
          for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i < j; i++) {
              double d = 0;
              for (int k = 0; k < K; k++) d += Q[(size_t)k * b + i] * Q[(size_t)k * b + j];
              for (int k = 0; k < K; k++) Q[(size_t)k * b + j] -= d * Q[(size_t)k * b + i];
              R[(size_t)i * b + j] += d;
            }
          double nrm = 0;
          for (int k = 0; k < K; k++) nrm += Q[(size_t)k * b + j] * Q[(size_t)k * b + j];
          nrm = std::sqrt(nrm);
          R[(size_t)j * b + j] = nrm;
          for (int k = 0; k < K; k++) Q[(size_t)k * b + j] /= nrm;
        }
        // pinv = diag(sc) R^-1 Q^T
        std::vector<double>& P = pinv[basis][n];
        P.assign((size_t)b * K, 0.0);
        for (int k = 0; k < K; k++) {
          // solve R x = Q^T e_k by back substitution
          std::vector<double> x(b);
          for (int i = b - 1; i >= 0; i--) {
            double v = Q[(size_t)k * b + i];
            for (int j = i + 1; j < b; j++) v -= R[(size_t)i * b + j] * x[j];
            x[i] = v / R[(size_t)i * b + i];
          }
          for (int i = 0; i < b; i++) P[(size_t)i * K + k] = sc[i] * x[i];
        }
      }
    }
  }

  // Rotation of basis `basis` for frame change x' = Q3 x, degrees 0..pr,
  // written as degree blocks into out (rot_size(pr) elements).
  void rotation(int basis, int pr, const double Q3[9], double* out) const {
    std::vector<std::vector<cplx>> tab(K);
    for (int k = 0; k < K; k++) {
      const double* x = &pts[3 * k];
      // back-rotated point y = Q3^T x
      double y[3];
      for (int i = 0; i < 3; i++) y[i] = Q3[i] * x[0] + Q3[3 + i] * x[1] + Q3[6 + i] * x[2];
      tab[k].resize(ncoef(pr));
      if (basis == 0)
        irregular_harmonics(pr, y[0], y[1], y[2], tab[k].data());
      else
        regular_harmonics(pr, y[0], y[1], y[2], tab[k].data());
    }
    for (int n = 0; n <= pr; n++) {
      const int b = 2 * n + 1, bb = 2 * n + 2;
      double* blk = out + rot_block_off(n);
      std::fill(blk, blk + (size_t)bb * bb, 0.0);
      const std::vector<double>& P = pinv[basis][n];
      std::vector<double> g(K);
      for (int j = 0; j < b; j++) {  // input slot
        const int sj = j == 0 ? 0 : j + 1;
        for (int k = 0; k < K; k++) g[k] = slot_value(basis, tab[k].data(), n, sj);
        for (int i = 0; i < b; i++) {  // output slot
          const int si = i == 0 ? 0 : i + 1;
          double v = 0;
          const double* Pi = &P[(size_t)i * K];
          for (int k = 0; k < K; k++) v += Pi[k] * g[k];
          blk[(size_t)si * bb + sj] = v;
        }
      }
    }
  }
};

// frame rotation with Q3 d = |d| e_z (rows u1, u2, d^)
void frame_for(const double d[3], double Q3[9]) {
  double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double u3[3] = {d[0] / r, d[1] / r, d[2] / r};
  if (std::fabs(u3[0]) < 1e-14 && std::fabs(u3[1]) < 1e-14) {
    double s = u3[2] > 0 ? 1.0 : -1.0;  // identity, or a half turn about x
    const double q[9] = {1, 0, 0, 0, s, 0, 0, 0, s};
    for (int i = 0; i < 9; i++) Q3[i] = q[i];
    return;
  }
  double u1[3] = {-u3[1], u3[0], 0.0};  // e_z x d^
  double n1 = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1]);
  u1[0] /= n1;
  u1[1] /= n1;
  double u2[3] = {u3[1] * u1[2] - u3[2] * u1[1], u3[2] * u1[0] - u3[0] * u1[2], u3[0] * u1[1] - u3[1] * u1[0]};
  for (int i = 0; i < 3; i++) {
    Q3[i] = u1[i];
    Q3[3 + i] = u2[i];
    Q3[6 + i] = u3[i];
  }
}

// shift along z by rho of `kind` truncated at p, order blocks into out
void zshift(int kind, int p, double rho, double* out) {
  std::vector<cplx> tab(ncoef(2 * p + 1));
  if (kind == 0)
    irregular_harmonics(2 * p, 0.0, 0.0, rho, tab.data());
  else
    regular_harmonics(p, 0.0, 0.0, rho, tab.data());
  for (int m = 0; m <= p; m++) {
    const int bz = 2 * (p - m + 1);
    double* blk = out + z_block_off(p, m);
    for (int n = m; n <= p; n++)
      for (int k = m; k <= p; k++) {
        double rr, ri, ir, ii;
        op_entry(kind, tab.data(), cidx(n, m), cidx(k, m), &rr, &ri, &ir, &ii);
        const int a = 2 * (n - m), c = 2 * (k - m);
        blk[(size_t)a * bz + c] = rr;
        blk[(size_t)a * bz + c + 1] = ri;
        blk[(size_t)(a + 1) * bz + c] = ir;
        blk[(size_t)(a + 1) * bz + c + 1] = ii;
      }
  }
}

template <class F>
void parallel_for(int n, F f) {
  int nt = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  nt = std::min(nt, std::max(n, 1));
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t]() {
      for (int i = t; i < n; i += nt) f(i);
    });
  for (auto& x : th) x.join();
}

}  // namespace

void build_factored_ops(int pmax, const std::vector<int>& kinds, const std::vector<int>& orders,
                        const std::vector<double>& offsets, std::vector<RotOp>& ops,
                        std::vector<double>& pool) {
  Fitter F;
  F.init(pmax);
  const int ng = (int)kinds.size();
  ops.resize(ng);
  long long off = 0;
  for (int g = 0; g < ng; g++) {
    const int p = orders[g];
    ops[g].p = p;
    ops[g].fw = off;
    off += rot_size(p);
    ops[g].z = off;
    off += z_size(p);
    ops[g].bk = off;
    off += rot_size(p);
  }
  pool.assign((size_t)off, 0.0);
  parallel_for(ng, [&](int g) {
    const int kind = kinds[g], p = orders[g];
    const double* d = &offsets[3 * g];
    double Q3[9], Qt[9];
    frame_for(d, Q3);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) Qt[3 * i + j] = Q3[3 * j + i];
    const double rho = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    // input basis of the forward rotation, output basis of the backward one
    const int bin = kind == 2 ? 1 : 0, bout = kind == 1 ? 0 : 1;
    F.rotation(bin, p, Q3, &pool[ops[g].fw]);
    zshift(kind, p, rho, &pool[ops[g].z]);
    F.rotation(bout, p, Qt, &pool[ops[g].bk]);
  });
}

void normalise_factored_ops(const std::vector<int>& kinds, const std::vector<RotOp>& ops,
                            const std::vector<double>& pool, const std::vector<double>& w,
                            std::vector<float>& out) {
  out.assign(pool.size(), 0.0f);
  parallel_for((int)ops.size(), [&](int g) {
    const RotOp& o = ops[g];
    const int kind = kinds[g], p = o.p;
    // scale factors: multipole rows x w, local rows / w (columns inverse)
    auto rs = [&](bool local, int row) { return local ? 1.0 / w[row] : w[row]; };
    const bool fw_in_local = kind == 2, z_in_local = kind == 2, z_out_local = kind != 1,
               bk_local = kind != 1;
    for (int n = 0; n <= p; n++) {
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      for (int i = 0; i < bb; i++)
        for (int j = 0; j < bb; j++) {
          size_t q = (size_t)i * bb + j;
          out[o.fw + rot_block_off(n) + q] =
              (float)(pool[o.fw + rot_block_off(n) + q] * rs(fw_in_local, r0 + i) / rs(fw_in_local, r0 + j));
          out[o.bk + rot_block_off(n) + q] =
              (float)(pool[o.bk + rot_block_off(n) + q] * rs(bk_local, r0 + i) / rs(bk_local, r0 + j));
        }
    }
    for (int m = 0; m <= p; m++) {
      const int bz = 2 * (p - m + 1);
      for (int a = 0; a < bz; a++)
        for (int c = 0; c < bz; c++) {
          const int ra = 2 * cidx(m + a / 2, m) + (a & 1), rc = 2 * cidx(m + c / 2, m) + (c & 1);
          size_t q = (size_t)z_block_off(p, m) + (size_t)a * bz + c;
          out[o.z + q] = (float)(pool[o.z + q] * rs(z_out_local, ra) / rs(z_in_local, rc));
        }
    }
  });
}

void column_major_factored(const std::vector<RotOp>& ops, std::vector<double>& pool) {
  parallel_for((int)ops.size(), [&](int g) {
    const RotOp& o = ops[g];
    const int p = o.p;
    std::vector<double> tmp;
    auto tr = [&](long long off, int b) {
      tmp.assign(pool.begin() + off, pool.begin() + off + (size_t)b * b);
      for (int i = 0; i < b; i++)
        for (int j = 0; j < b; j++) pool[off + (size_t)j * b + i] = tmp[(size_t)i * b + j];
    };
    for (int n = 0; n <= p; n++) {
      tr(o.fw + rot_block_off(n), 2 * n + 2);
      tr(o.bk + rot_block_off(n), 2 * n + 2);
    }
    for (int m = 0; m <= p; m++) tr(o.z + z_block_off(p, m), 2 * (p - m + 1));
  });
}

double check_factored_ops(const std::vector<int>& kinds, const std::vector<int>& orders,
                          const std::vector<double>& offsets, const std::vector<RotOp>& ops,
                          const std::vector<double>& pool, int stride) {
  double worst = 0;
  std::mt19937_64 rng(7);
  std::normal_distribution<double> N01;
  for (int g = 0; g < (int)kinds.size(); g += std::max(stride, 1)) {
    const int kind = kinds[g], p = orders[g], nc = ncoef(p), dim = 2 * nc;
    const double* d = &offsets[3 * g];
    std::vector<cplx> tab(ncoef(2 * p + 1));
    if (kind == 0)
      irregular_harmonics(2 * p, d[0], d[1], d[2], tab.data());
    else
      regular_harmonics(p, d[0], d[1], d[2], tab.data());
    // a random expansion of a real field (Im of m = 0 is zero), O(1) in the
    // normalised basis (multipole x w, local / w, w = sqrt((n+m)!(n-m)!)),
    // where the harmonics are O(1) and the error measure is meaningful
    std::vector<double> v(dim), a(dim, 0.0), f(dim, 0.0), z(dim, 0.0), b(dim, 0.0), wr(dim);
    for (int n = 0; n <= p; n++)
      for (int m = 0; m <= n; m++)
        wr[2 * cidx(n, m)] = wr[2 * cidx(n, m) + 1] =
            std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
    const bool in_local = kind == 2, out_local = kind != 1;
    for (int q = 0; q < dim; q++) v[q] = N01(rng) * (in_local ? wr[q] : 1.0 / wr[q]);
    for (int n = 0; n <= p; n++) v[2 * cidx(n, 0) + 1] = 0.0;
    for (int r = 0; r < nc; r++)
      for (int c = 0; c < nc; c++) {
        double rr, ri, ir, ii;
        op_entry(kind, tab.data(), r, c, &rr, &ri, &ir, &ii);
        a[2 * r] += rr * v[2 * c] + ri * v[2 * c + 1];
        a[2 * r + 1] += ir * v[2 * c] + ii * v[2 * c + 1];
      }
    const RotOp& o = ops[g];
    for (int n = 0; n <= p; n++) {
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      const double* B = &pool[o.fw + rot_block_off(n)];
      for (int i = 0; i < bb; i++)
        for (int j = 0; j < bb; j++) f[r0 + i] += B[(size_t)i * bb + j] * v[r0 + j];
    }
    for (int m = 0; m <= p; m++) {
      const int bz = 2 * (p - m + 1);
      const double* Z = &pool[o.z + z_block_off(p, m)];
      for (int a_ = 0; a_ < bz; a_++)
        for (int c = 0; c < bz; c++)
          z[2 * cidx(m + a_ / 2, m) + (a_ & 1)] += Z[(size_t)a_ * bz + c] * f[2 * cidx(m + c / 2, m) + (c & 1)];
    }
    for (int n = 0; n <= p; n++) {
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      const double* B = &pool[o.bk + rot_block_off(n)];
      for (int i = 0; i < bb; i++)
        for (int j = 0; j < bb; j++) b[r0 + i] += B[(size_t)i * bb + j] * z[r0 + j];
    }
    double num = 0, den = 0;
    for (int n = 0; n <= p; n++)
      for (int m = 0; m <= n; m++)
        for (int part = 0; part < 2; part++) {
          if (m == 0 && part == 1) continue;  // not part of a real field
          const int q = 2 * cidx(n, m) + part;
          const double sc = out_local ? 1.0 / wr[q] : wr[q];
          num += (a[q] - b[q]) * (a[q] - b[q]) * sc * sc;
          den += a[q] * a[q] * sc * sc;
        }
    worst = std::max(worst, std::sqrt(num / std::max(den, 1e-300)));
  }
  return worst;
}

// ------------------------------------------------------- parity-split form
// The frame change of a translation is taken as Q = Ry(-theta) Rz(-phi)
// (theta, phi the polar angles of the offset), so the coefficient map is
// M(Q) = M(Ry) M(Rz).  M(Rz) mixes only the (re, im) pair of each (n, m): a
// 2 x 2 matrix per order m, the same for every degree.  A rotation about y
// commutes with the reflection y -> -y, so M(Ry) never mixes the re (cos m
// phi) and im (sin m phi) parts: per degree n an (n+1) x (n+1) re block and
// an n x n im block.  The shift along z commutes with both, so it is an
// re block and an im block per order m as well.  Per pair and column this is
// about 2 p^3 multiply-adds against the 4 p^3 of the full (2n+2)^2 and
// (2(p-m+1))^2 blocks.

namespace {

// The parity-split factors of one group, factorial basis, double.
// Block b of r rows is stored row-major as re[r*r], then im[r*r] (im row and
// column 0 zero in the rotations: m = 0 has no sin part; the shift's im block
// of order 0 zero).
struct SplitHost {
  int p = 0;
  std::vector<double> rz[2];  // [fw, bk]: 4 per order m (re<-re, re<-im, im<-re, im<-im)
  std::vector<std::vector<double>> ry[2];  // [fw, bk][n]: 2 (n+1)^2
  std::vector<std::vector<double>> z;      // [m]: 2 (p-m+1)^2
  double cross = 0;  // largest coupling dropped by the split (relative)
};

void rot_y(double a, double Q[9]) {  // frame change x' = Ry(a) x
  const double c = std::cos(a), s = std::sin(a);
  const double q[9] = {c, 0, s, 0, 1, 0, -s, 0, c};
  for (int i = 0; i < 9; i++) Q[i] = q[i];
}
void rot_z(double a, double Q[9]) {  // frame change x' = Rz(a) x
  const double c = std::cos(a), s = std::sin(a);
  const double q[9] = {c, -s, 0, s, c, 0, 0, 0, 1};
  for (int i = 0; i < 9; i++) Q[i] = q[i];
}

// degree blocks of a fitted rotation (slot order 2m + part) -> re / im
// blocks; the largest cross term relative to the block's largest entry
double split_rotation(const std::vector<double>& full, int p, std::vector<std::vector<double>>& out) {
  double cross = 0;
  out.assign(p + 1, {});
  for (int n = 0; n <= p; n++) {
    const int bb = 2 * n + 2, r = n + 1;
    const double* B = &full[rot_block_off(n)];
    std::vector<double>& o = out[n];
    o.assign(2 * (size_t)r * r, 0.0);
    double big = 0, cr = 0;
    for (int i = 0; i < r; i++)
      for (int k = 0; k < r; k++) {
        o[(size_t)i * r + k] = B[(size_t)(2 * i) * bb + 2 * k];
        if (i > 0 && k > 0) o[(size_t)r * r + (size_t)i * r + k] = B[(size_t)(2 * i + 1) * bb + 2 * k + 1];
        big = std::max(big, std::fabs(B[(size_t)(2 * i) * bb + 2 * k]));
        cr = std::max({cr, std::fabs(B[(size_t)(2 * i) * bb + 2 * k + 1]), std::fabs(B[(size_t)(2 * i + 1) * bb + 2 * k])});
      }
    cross = std::max(cross, cr / std::max(big, 1e-300));
  }
  return cross;
}

// the 2 x 2 per order of a fitted rotation about z (taken from degree p; the
// other degrees and every off-order entry checked)
double split_rz(const std::vector<double>& full, int p, std::vector<double>& out) {
  out.assign(4 * (size_t)(p + 1), 0.0);
  double dev = 0;
  for (int n = 0; n <= p; n++) {
    const int bb = 2 * n + 2;
    const double* B = &full[rot_block_off(n)];
    for (int i = 0; i < bb; i++)
      for (int k = 0; k < bb; k++) {
        const double v = B[(size_t)i * bb + k];
        if ((i >> 1) != (k >> 1)) {
          dev = std::max(dev, std::fabs(v));
          continue;
        }
        const int m = i >> 1, q = 2 * (i & 1) + (k & 1);
        if (m == 0 && (i == 1 || k == 1)) continue;  // inactive slot
        if (n == p)
          out[4 * m + q] = v;
      }
  }
  for (int n = 0; n < p; n++) {
    const int bb = 2 * n + 2;
    const double* B = &full[rot_block_off(n)];
    for (int m = 0; m <= n; m++)
      for (int q = 0; q < 4; q++) {
        if (m == 0 && q != 0) continue;
        const int i = 2 * m + (q >> 1), k = 2 * m + (q & 1);
        dev = std::max(dev, std::fabs(B[(size_t)i * bb + k] - out[4 * m + q]));
      }
  }
  return dev;
}

void build_split_host(int kind, int p, const double d[3], const Fitter& F, SplitHost& S) {
  S.p = p;
  const double rho = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double th = std::acos(std::max(-1.0, std::min(1.0, d[2] / rho)));
  const double ph = (d[0] == 0.0 && d[1] == 0.0) ? 0.0 : std::atan2(d[1], d[0]);
  double Qz[9], Qy[9], Qzt[9], Qyt[9];
  rot_z(-ph, Qz);
  rot_y(-th, Qy);
  rot_z(ph, Qzt);
  rot_y(th, Qyt);
  const int bin = kind == 2 ? 1 : 0, bout = kind == 1 ? 0 : 1;
  std::vector<double> full(rot_size(p));
  double cross = 0;
  F.rotation(bin, p, Qz, full.data());
  cross = std::max(cross, split_rz(full, p, S.rz[0]));
  F.rotation(bin, p, Qy, full.data());
  cross = std::max(cross, split_rotation(full, p, S.ry[0]));
  F.rotation(bout, p, Qyt, full.data());
  cross = std::max(cross, split_rotation(full, p, S.ry[1]));
  F.rotation(bout, p, Qzt, full.data());
  cross = std::max(cross, split_rz(full, p, S.rz[1]));
  std::vector<double> zf(z_size(p));
  zshift(kind, p, rho, zf.data());
  S.z.assign(p + 1, {});
  for (int m = 0; m <= p; m++) {
    const int r = p - m + 1, bz = 2 * r;
    const double* B = &zf[z_block_off(p, m)];
    std::vector<double>& o = S.z[m];
    o.assign(2 * (size_t)r * r, 0.0);
    double big = 0, cr = 0;
    for (int i = 0; i < r; i++)
      for (int k = 0; k < r; k++) {
        o[(size_t)i * r + k] = B[(size_t)(2 * i) * bz + 2 * k];
        if (m > 0) o[(size_t)r * r + (size_t)i * r + k] = B[(size_t)(2 * i + 1) * bz + 2 * k + 1];
        big = std::max(big, std::fabs(B[(size_t)(2 * i) * bz + 2 * k]));
        cr = std::max({cr, std::fabs(B[(size_t)(2 * i) * bz + 2 * k + 1]), std::fabs(B[(size_t)(2 * i + 1) * bz + 2 * k])});
      }
    cross = std::max(cross, cr / std::max(big, 1e-300));
  }
  S.cross = cross;
}

// y = Bk Z Fw v of the split factors (v, y: 2 ncoef(p) in storage order)
void apply_split_host(const SplitHost& S, const std::vector<double>& v, std::vector<double>& y) {
  const int p = S.p, dim = 2 * ncoef(p);
  std::vector<double> a(v), b(dim, 0.0);
  auto rz = [&](const std::vector<double>& R, std::vector<double>& x) {
    for (int n = 0; n <= p; n++)
      for (int m = 0; m <= n; m++) {
        const int c = 2 * cidx(n, m);
        const double re = x[c], im = x[c + 1];
        x[c] = R[4 * m] * re + R[4 * m + 1] * im;
        x[c + 1] = R[4 * m + 2] * re + R[4 * m + 3] * im;
      }
  };
  auto ry = [&](const std::vector<std::vector<double>>& Bl, std::vector<double>& x) {
    std::vector<double> t(x);
    for (int n = 0; n <= p; n++) {
      const int r = n + 1;
      for (int i = 0; i < r; i++) {
        double sr = 0, si = 0;
        for (int k = 0; k < r; k++) {
          sr += Bl[n][(size_t)i * r + k] * t[2 * cidx(n, k)];
          si += Bl[n][(size_t)r * r + (size_t)i * r + k] * t[2 * cidx(n, k) + 1];
        }
        x[2 * cidx(n, i)] = sr;
        x[2 * cidx(n, i) + 1] = si;
      }
    }
  };
  rz(S.rz[0], a);
  ry(S.ry[0], a);
  for (int m = 0; m <= p; m++) {
    const int r = p - m + 1;
    for (int i = 0; i < r; i++) {
      double sr = 0, si = 0;
      for (int k = 0; k < r; k++) {
        sr += S.z[m][(size_t)i * r + k] * a[2 * cidx(m + k, m)];
        si += S.z[m][(size_t)r * r + (size_t)i * r + k] * a[2 * cidx(m + k, m) + 1];
      }
      b[2 * cidx(m + i, m)] = sr;
      b[2 * cidx(m + i, m) + 1] = si;
    }
  }
  ry(S.ry[1], b);
  rz(S.rz[1], b);
  y = b;
}

}  // namespace

// floats of the split blocks of r = 1..R rows: r operator columns and one
// zero column, ceil(r/2) float4 each
EFMM_HD constexpr long long rots_blocks(int R) {
  long long s = 0;
  for (int r = 1; r <= R; r++) s += 4LL * (r + 1) * ((r + 1) / 2);
  return s;
}
long long rots_group_size(int p) { return 8LL * (p + 1) + 3 * rots_blocks(p + 1); }

void build_split_ops(const std::vector<int>& kinds, const std::vector<int>& orders,
                     const std::vector<double>& offsets, const std::vector<double>& w,
                     std::vector<RotSOp>& ops, std::vector<float>& pool) {
  const int ng = (int)kinds.size();
  int pmax = 0;
  for (int q : orders) pmax = std::max(pmax, q);
  Fitter F;
  F.init(pmax);
  ops.resize(ng);
  long long off = 0;
  for (int g = 0; g < ng; g++) {
    ops[g].p = orders[g];
    ops[g].pad = 0;
    ops[g].base = off;
    off += rots_group_size(orders[g]);
  }
  pool.assign((size_t)off, 0.0f);
  parallel_for(ng, [&](int g) {
    const int kind = kinds[g], p = orders[g];
    SplitHost S;
    build_split_host(kind, p, &offsets[3 * g], F, S);
    // normalised basis: multipole rows x w, local rows / w (columns inverse)
    auto rs = [&](bool local, int n, int m) {
      const double v = w[2 * cidx(n, m)];
      return local ? 1.0 / v : v;
    };
    const bool fw_local = kind == 2, z_in_local = kind == 2, z_out_local = kind != 1, bk_local = kind != 1;
    float* o = &pool[ops[g].base];
    for (int s = 0; s < 2; s++) {
      float* rz = s == 0 ? o : o + 4 * (p + 1) + 3 * rots_blocks(p + 1);
      for (int q = 0; q < 4 * (p + 1); q++) rz[q] = (float)S.rz[s][q];
    }
    // a block of r rows: column k holds ceil(r/2) float4 (re[2j][k],
    // im[2j][k], re[2j+1][k], im[2j+1][k]); column r stays zero
    auto pack = [&](float* dst, const std::vector<double>& B, int r, auto scale) {
      const int h = (r + 1) / 2;
      for (int k = 0; k < r; k++)
        for (int j = 0; j < h; j++)
          for (int e = 0; e < 4; e++) {
            const int i = 2 * j + (e >> 1), part = e & 1;
            double v = 0;
            if (i < r) v = B[(size_t)part * r * r + (size_t)i * r + k] * scale(i, k);
            dst[((size_t)k * h + j) * 4 + e] = (float)v;
          }
    };
    float* ryf = o + 4 * (p + 1);
    float* zb = ryf + rots_blocks(p + 1);
    float* ryb = zb + rots_blocks(p + 1);
    for (int n = 0; n <= p; n++) {
      pack(ryf + rots_blocks(n), S.ry[0][n], n + 1,
           [&](int i, int k) { return rs(fw_local, n, i) / rs(fw_local, n, k); });
      pack(ryb + rots_blocks(n), S.ry[1][n], n + 1,
           [&](int i, int k) { return rs(bk_local, n, i) / rs(bk_local, n, k); });
    }
    for (int m = 0; m <= p; m++)
      pack(zb + rots_blocks(p + 1) - rots_blocks(p + 1 - m), S.z[m], p - m + 1,
           [&](int i, int k) { return rs(z_out_local, m + i, m) / rs(z_in_local, m + k, m); });
  });
}

// ------------------------------ M2L of the half-space kernel U, parity split
// U is unchanged by rotations about z and by the reflection y -> -y, so its
// M2L operator for an offset d = (rho cos phi, rho sin phi, dz) is
//   T(d) = M_out(Rz(phi)) T(d0) M_in(Rz(-phi)),  d0 = (rho, 0, dz),
// and T(d0) (offset in the xz plane) never mixes the re and im parts: an
// ncoef x ncoef re block and an im block (row and column of order 0 zero).
// Groups with the same (rho, dz, order) share their blocks.

namespace {
// T(d) of the U kernel at order p in the factorial basis (rows and columns
// 2 ncoef, row-major), from the same J table and entries as the device builder
void u_dense(int p, const double d[3], std::vector<double>& T) {
  const int nc = ncoef(p), dim = 2 * nc;
  std::vector<cplx> J(ncoef(2 * p + 1));
  u_harmonics(2 * p, d[0], d[1], d[2], J.data());
  T.assign((size_t)dim * dim, 0.0);
  for (int r = 0; r < nc; r++)
    for (int c = 0; c < nc; c++) {
      double rr, ri, ir, ii;
      op_entry(0, J.data(), r, c, &rr, &ri, &ir, &ii);
      T[(size_t)(2 * r) * dim + 2 * c] = rr;
      T[(size_t)(2 * r) * dim + 2 * c + 1] = ri;
      T[(size_t)(2 * r + 1) * dim + 2 * c] = ir;
      T[(size_t)(2 * r + 1) * dim + 2 * c + 1] = ii;
    }
}
}  // namespace

void build_usplit_ops(const std::vector<int>& orders, const std::vector<double>& offsets, const std::vector<double>& w,
                      std::vector<USOp>& ops, std::vector<float>& pool, double* cross) {
  const int ng = (int)orders.size();
  int pmax = 0;
  for (int q : orders) pmax = std::max(pmax, q);
  Fitter F;
  F.init(pmax);
  // distinct (rho^2, dz, order): the blocks
  std::vector<long long> key(ng);
  std::vector<int> bidx(ng);
  std::vector<long long> bkeys;
  std::vector<int> bg;  // a group of each block
  for (int g = 0; g < ng; g++) {
    const double* d = &offsets[3 * g];
    const long long r2 = llround(d[0] * d[0] + d[1] * d[1]);
    key[g] = (r2 * 64 + llround(d[2]) + 32) * 64 + orders[g];
    int b = -1;
    for (size_t q = 0; q < bkeys.size(); q++)
      if (bkeys[q] == key[g]) b = (int)q;
    if (b < 0) {
      b = (int)bkeys.size();
      bkeys.push_back(key[g]);
      bg.push_back(g);
    }
    bidx[g] = b;
  }
  const int nbk = (int)bkeys.size();
  ops.resize(ng);
  long long off = 0;
  std::vector<long long> boff(nbk);
  for (int b = 0; b < nbk; b++) {
    const int nc = ncoef(orders[bg[b]]), ld = (nc + 3) & ~3;
    boff[b] = off;
    off += 2LL * nc * ld;
  }
  for (int g = 0; g < ng; g++) {
    const int nc = ncoef(orders[g]), ld = (nc + 3) & ~3;
    ops[g].p = orders[g];
    ops[g].ld = ld;
    ops[g].re = boff[bidx[g]];
    ops[g].im = boff[bidx[g]] + (long long)nc * ld;
    ops[g].rzi = off;
    off += 4LL * (orders[g] + 1);
    ops[g].rzo = off;
    off += 4LL * (orders[g] + 1);
  }
  pool.assign((size_t)off, 0.0f);
  std::vector<double> bcross(nbk, 0.0);
  parallel_for(nbk, [&](int b) {
    const int g = bg[b], p = orders[g], nc = ncoef(p), dim = 2 * nc, ld = ops[g].ld;
    const double* d = &offsets[3 * g];
    const double d0[3] = {std::sqrt(d[0] * d[0] + d[1] * d[1]), 0.0, d[2]};
    std::vector<double> T;
    u_dense(p, d0, T);
    double big = 0, cr = 0;
    float* re = &pool[ops[g].re];
    float* im = &pool[ops[g].im];
    std::vector<int> mof(nc);
    for (int n = 0; n <= p; n++)
      for (int m = 0; m <= n; m++) mof[cidx(n, m)] = m;
    for (int r = 0; r < nc; r++)
      for (int c = 0; c < nc; c++) {
        const double s = 1.0 / (w[2 * r] * w[2 * c]);  // local rows / w, multipole columns x w
        const double a = T[(size_t)(2 * r) * dim + 2 * c], e = T[(size_t)(2 * r + 1) * dim + 2 * c + 1];
        re[(size_t)r * ld + c] = (float)(a * s);
        if (mof[r] > 0 && mof[c] > 0) im[(size_t)r * ld + c] = (float)(e * s);
        big = std::max(big, std::fabs(a * s));
        cr = std::max({cr, std::fabs(T[(size_t)(2 * r) * dim + 2 * c + 1] * s),
                       std::fabs(T[(size_t)(2 * r + 1) * dim + 2 * c] * s)});
      }
    bcross[b] = cr / std::max(big, 1e-300);
  });
  parallel_for(ng, [&](int g) {
    const int p = orders[g];
    const double* d = &offsets[3 * g];
    const double ph = (d[0] == 0.0 && d[1] == 0.0) ? 0.0 : std::atan2(d[1], d[0]);
    double Qz[9], Qzt[9];
    rot_z(-ph, Qz);
    rot_z(ph, Qzt);
    std::vector<double> full(rot_size(p)), rz;
    F.rotation(0, p, Qz, full.data());
    split_rz(full, p, rz);
    for (int q = 0; q < 4 * (p + 1); q++) pool[ops[g].rzi + q] = (float)rz[q];
    F.rotation(1, p, Qzt, full.data());
    split_rz(full, p, rz);
    for (int q = 0; q < 4 * (p + 1); q++) pool[ops[g].rzo + q] = (float)rz[q];
  });
  if (cross) {
    *cross = 0;
    for (double c : bcross) *cross = std::max(*cross, c);
  }
}

// ------------------------------------------------------------------ kernel
// One CTA per tile of NCT columns of one group.  The columns are staged in
// shared memory (rows x NCT), rotated (X -> Y), shifted (Y -> X), rotated
// back (X -> Y) and added to the destinations (ROT_THREADS threads: the
// operator loads come from L2, so more warps hide more of their latency).  The device pool stores every
// block column-major, so the 8 coefficients a warp works on read one
// contiguous operator segment per k; a lane computes the re and im rows of
// one coefficient for G consecutive columns (G = 4 FP32, 2 FP64).
template <class T>
struct Vec4T;
template <>
struct Vec4T<float> {
  static __device__ __forceinline__ void ld(const float* p, float* v) {
    float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  }
  static __device__ __forceinline__ void st(float* p, const float* v) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct Vec4T<double> {
  static __device__ __forceinline__ void ld(const double* p, double* v) {
    double2 q = *reinterpret_cast<const double2*>(p);
    v[0] = q.x; v[1] = q.y;
  }
  static __device__ __forceinline__ void st(double* p, const double* v) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  }
};

__device__ __forceinline__ void coef_nm(int cc, int& n, int& m) {
  n = (int)((sqrt(8.0 * cc + 1.0) - 1.0) * 0.5);
  while ((n + 1) * (n + 2) / 2 <= cc) n++;
  while (n * (n + 1) / 2 > cc) n--;
  m = cc - n * (n + 1) / 2;
}

constexpr int ROT_THREADS = 512;

// a0 += wx x, a1 += wy x over G columns (paired FP32 FMAs measured slower
// here than in k_translate_rot_w: this kernel is not issue-bound)
template <class T, int G>
__device__ __forceinline__ void fma_rows(T* a0, T* a1, T wx, T wy, const T* x) {
#pragma unroll
  for (int g = 0; g < G; g++) {
    a0[g] += wx * x[g];
    a1[g] += wy * x[g];
  }
}

template <class T, int NCT>
__global__ void __launch_bounds__(ROT_THREADS)
k_translate_rot(const TransTask* __restrict__ tasks, const TransPair* __restrict__ pairs,
                const RotOp* __restrict__ ops, const T* __restrict__ pool, int D, int C,
                const T* __restrict__ src, T* __restrict__ dst) {
  constexpr int G = NCT / 4;  // columns per lane
  using V = Vec4T<T>;
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char rt_smem[];
  const TransTask t = tasks[blockIdx.x];
  const RotOp op = ops[t.group];
  const int p = op.p, dim = (p + 1) * (p + 2), nc = dim / 2;
  T* X = reinterpret_cast<T*>(rt_smem);
  T* Y = X + (size_t)dim * NCT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // stage: thread (row r, column group) loads G columns, one vector store
  {
    const T* sp[NCT];
#pragma unroll
    for (int j = 0; j < NCT; j++) {
      const int col = t.col0 + j;
      sp[j] = nullptr;
      if (col < t.ncols) {
        const TransPair pr = pairs[t.pair0 + col / C];
        sp[j] = src + ((size_t)pr.src * C + col % C) * D;
      }
    }
    for (int q = tid; q < dim * 4; q += ROT_THREADS) {
      const int r = q % dim, cg = q / dim;
      T v[G];
#pragma unroll
      for (int g = 0; g < G; g++) v[g] = sp[cg * G + g] ? sp[cg * G + g][r] : T(0);
      V::st(X + (size_t)r * NCT + cg * G, v);
    }
  }
  __syncthreads();
  const int sub = lane >> 2, cg = lane & 3;  // coefficient within the warp's 8, column group
  // rotation stage (degree blocks), coefficients in storage order
  auto rotate = [&](const T* in, T* out, long long base) {
    for (int c0 = warp * 8; c0 < nc; c0 += ROT_THREADS / 4) {
      const int cc = c0 + sub;
      if (cc >= nc) continue;
      int n, m;
      coef_nm(cc, n, m);
      const int r0 = n * (n + 1), bb = 2 * n + 2;
      const T* o = pool + base + rot_block_off(n) + 2 * m;  // column-major: (row, k) at k*bb + row
      T a0[G], a1[G];
#pragma unroll
      for (int g = 0; g < G; g++) a0[g] = a1[g] = T(0);
      // bb = 2n + 2 is even: two k per step, operator pairs as vectors,
      // UNR steps of loads issued before their products
      constexpr int UNR = 4;
      int k = 0;
      for (; k + 2 * UNR <= bb; k += 2 * UNR) {
        V2 w[2 * UNR];
#pragma unroll
        for (int u = 0; u < 2 * UNR; u++) w[u] = *reinterpret_cast<const V2*>(o + (size_t)(k + u) * bb);
#pragma unroll
        for (int u = 0; u < 2 * UNR; u++) {
          T xv[G];
          V::ld(in + (size_t)(r0 + k + u) * NCT + cg * G, xv);
          fma_rows<T, G>(a0, a1, w[u].x, w[u].y, xv);
        }
      }
      for (; k < bb; k++) {
        const V2 w = *reinterpret_cast<const V2*>(o + (size_t)k * bb);
        T xv[G];
        V::ld(in + (size_t)(r0 + k) * NCT + cg * G, xv);
        fma_rows<T, G>(a0, a1, w.x, w.y, xv);
      }
      V::st(out + (size_t)(2 * cc) * NCT + cg * G, a0);
      V::st(out + (size_t)(2 * cc + 1) * NCT + cg * G, a1);
    }
  };
  rotate(X, Y, op.fw);
  __syncthreads();
  // shift along z: coefficients in order-major order (m, then n = m..p)
  for (int q0 = warp * 8; q0 < nc; q0 += ROT_THREADS / 4) {
    const int q = q0 + sub;
    if (q >= nc) continue;
    int m = 0, start = 0;
    while (start + (p - m + 1) <= q) {
      start += p - m + 1;
      m++;
    }
    const int n = m + (q - start);
    const int bz = 2 * (p - m + 1), a = 2 * (n - m);
    const T* o = pool + op.z + z_block_off(p, m) + a;  // column-major: (row, col) at col*bz + row
    T a0[G], a1[G];
#pragma unroll
    for (int g = 0; g < G; g++) a0[g] = a1[g] = T(0);
    int k = m;
    constexpr int UNZ = 4;
    for (; k + UNZ <= p + 1; k += UNZ) {
      V2 wr[UNZ], wi[UNZ];
#pragma unroll
      for (int u = 0; u < UNZ; u++) {
        const int c = 2 * (k + u - m);
        wr[u] = *reinterpret_cast<const V2*>(o + (size_t)c * bz);
        wi[u] = *reinterpret_cast<const V2*>(o + (size_t)(c + 1) * bz);
      }
#pragma unroll
      for (int u = 0; u < UNZ; u++) {
        const int rk = 2 * ((k + u) * (k + u + 1) / 2 + m);
        T xr[G], xi[G];
        V::ld(Y + (size_t)rk * NCT + cg * G, xr);
        V::ld(Y + (size_t)(rk + 1) * NCT + cg * G, xi);
        fma_rows<T, G>(a0, a1, wr[u].x, wr[u].y, xr);
        fma_rows<T, G>(a0, a1, wi[u].x, wi[u].y, xi);
      }
    }
    for (; k <= p; k++) {
      const int c = 2 * (k - m);
      const V2 wr = *reinterpret_cast<const V2*>(o + (size_t)c * bz);
      const V2 wi = *reinterpret_cast<const V2*>(o + (size_t)(c + 1) * bz);
      const int rk = 2 * (k * (k + 1) / 2 + m);
      T xr[G], xi[G];
      V::ld(Y + (size_t)rk * NCT + cg * G, xr);
      V::ld(Y + (size_t)(rk + 1) * NCT + cg * G, xi);
      fma_rows<T, G>(a0, a1, wr.x, wr.y, xr);
      fma_rows<T, G>(a0, a1, wi.x, wi.y, xi);
    }
    const int cc = n * (n + 1) / 2 + m;
    V::st(X + (size_t)(2 * cc) * NCT + cg * G, a0);
    V::st(X + (size_t)(2 * cc + 1) * NCT + cg * G, a1);
  }
  __syncthreads();
  rotate(X, Y, op.bk);
  __syncthreads();
  for (int j = 0; j < NCT; j++) {
    const int col = t.col0 + j;
    if (col >= t.ncols) break;
    const TransPair pr = pairs[t.pair0 + col / C];
    T* dp = dst + ((size_t)pr.dst * C + col % C) * D;
    const T al = (T)pr.alpha;
    for (int r = tid; r < dim; r += ROT_THREADS) atomicAdd(dp + r, al * Y[(size_t)r * NCT + j]);
  }
}

// FP32 factored translations with one warp per degree block (rotations) or
// order block (shift along z), in place: the 16 columns of the task stay in
// one shared buffer X[row][16]; a warp owns whole blocks (lane l: output
// rows 2l, 2l + 1 of the block, all 16 columns in registers), reads its
// block's operator columns from global memory (one coalesced 8-byte load per
// lane and k) and the input rows of X as broadcasts, and writes its rows
// back after the block's reads (__syncwarp).  Blocks are spread over the
// warps by size (longest first).  For orders p <= 31 (blocks of <= 64 rows);
// half the shared memory of k_translate_rot, two CTAs of 12 warps per SM.
constexpr int ROTW_THREADS = 384, ROTW_NCT = 16, ROTW_PMAX = 31, ROTW_NW = ROTW_THREADS / 32;

// Warp of degree block n at order p (order block p - n of the shift): the
// blocks, (2n + 2)^2 entries each, spread largest first onto the least
// loaded warp; fixed per order, built at compile time.
struct RotwOwners {
  unsigned char o[ROTW_PMAX + 1][ROTW_PMAX + 1];
};
constexpr RotwOwners make_rotw_owners() {
  RotwOwners r{};
  for (int p = 0; p <= ROTW_PMAX; p++) {
    int load[ROTW_NW] = {};
    for (int n = p; n >= 0; n--) {
      int best = 0;
      for (int w = 1; w < ROTW_NW; w++)
        if (load[w] < load[best]) best = w;
      r.o[p][n] = (unsigned char)best;
      load[best] += (n + 1) * (n + 1);
    }
  }
  return r;
}
__constant__ RotwOwners c_rotw_owners = make_rotw_owners();
// shared memory: X [dim][16] floats, the source column offsets [16], then
// per warp two operator buffers of ROTW_CH columns of <= 64 rows
constexpr int ROTW_CH = 8;
__host__ __device__ inline size_t rotw_cbase_off(int dim) { return sizeof(float) * (size_t)dim * ROTW_NCT; }
__host__ __device__ inline size_t rotw_wbuf_off(int dim) { return rotw_cbase_off(dim) + 8 * ROTW_NCT; }
__host__ __device__ inline size_t rotw_smem(int dim) {
  return rotw_wbuf_off(dim) + sizeof(float) * (size_t)ROTW_NW * 2 * ROTW_CH * 64;
}

__global__ void __launch_bounds__(ROTW_THREADS, 2)
k_translate_rot_w(const TransTask* __restrict__ tasks, const TransPair* __restrict__ pairs,
                  const RotOp* __restrict__ ops, const float* __restrict__ pool, int D, int C,
                  const float* __restrict__ src, float* __restrict__ dst) {
  constexpr int NCT = ROTW_NCT, G = NCT / 4;
  extern __shared__ __align__(16) unsigned char rw_smem[];
  const TransTask t = tasks[blockIdx.x];
  const RotOp op = ops[t.group];
  const int p = op.p, dim = (p + 1) * (p + 2);
  float* X = reinterpret_cast<float*>(rw_smem);                                   // [dim][NCT]
  long long* cbase = reinterpret_cast<long long*>(rw_smem + rotw_cbase_off(dim));  // [NCT]: source columns
  const unsigned char* owner = c_rotw_owners.o[p];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < NCT) {
    const int col = t.col0 + tid;
    long long b = -1;
    if (col < t.ncols) {
      const TransPair pr = pairs[t.pair0 + col / C];
      b = ((long long)pr.src * C + col % C) * D;
    }
    cbase[tid] = b;
  }
  __syncthreads();
  for (int q = tid; q < dim * 4; q += ROTW_THREADS) {
    const int r = q % dim, cg = q / dim;
    float v[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
      const long long b = cbase[cg * G + g];
      v[g] = b >= 0 ? src[b + r] : 0.0f;
    }
    *reinterpret_cast<float4*>(X + (size_t)r * NCT + cg * G) = make_float4(v[0], v[1], v[2], v[3]);
  }
  __syncthreads();
  // accumulators: column pairs (2c, 2c + 1) packed in a float2, updated by
  // the paired FP32 FMA (__ffma2_rn: two correctly rounded FMAs in one
  // instruction, half the issue slots of the products)
  auto put_rows = [&](int ra, int rb, const float2* a0, const float2* a1) {
#pragma unroll
    for (int q = 0; q < NCT / 4; q++) {
      *reinterpret_cast<float4*>(X + (size_t)ra * NCT + 4 * q) =
          make_float4(a0[2 * q].x, a0[2 * q].y, a0[2 * q + 1].x, a0[2 * q + 1].y);
      *reinterpret_cast<float4*>(X + (size_t)rb * NCT + 4 * q) =
          make_float4(a1[2 * q].x, a1[2 * q].y, a1[2 * q + 1].x, a1[2 * q + 1].y);
    }
  };
  // the warp's operator columns, ROTW_CH at a time, copied asynchronously
  // into its two shared buffers (one chunk ahead of the products); a block's
  // columns are contiguous (column-major, ld = rows <= 64)
  float* wbuf = reinterpret_cast<float*>(rw_smem + rotw_wbuf_off(dim)) + (size_t)warp * 2 * ROTW_CH * 64;
  auto fetch = [&](const float* blk, int ld, int ncol, int chunk) {
    const int c0 = chunk * ROTW_CH, nbytes = 4 * min(ROTW_CH, ncol - c0) * ld;
    const float* g = blk + (size_t)c0 * ld;
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(wbuf + (chunk & 1) * ROTW_CH * 64));
    for (int b = 16 * lane; b < nbytes; b += 16 * 32) {
      const int nb = min(16, nbytes - b);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d + b), "l"(reinterpret_cast<const char*>(g) + b),
                   "r"(nb)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // one block product: rows 2 lane, 2 lane + 1 of the block (if < nrow),
  // columns kk < ncol of the operator (ld = nrow); the operator column pairs
  // of input row k are (2k, 2k + 1) for the shift (pair = true), else k
  auto block = [&](const float* blk, int nrow, int ncol, bool pair, auto xrow, float2* a0, float2* a1) {
    const bool act = 2 * lane < nrow;
    const int nch = (ncol + ROTW_CH - 1) / ROTW_CH;
    fetch(blk, nrow, ncol, 0);
    for (int ch = 0; ch < nch; ch++) {
      if (ch + 1 < nch)
        fetch(blk, nrow, ncol, ch + 1);
      else
        asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
      __syncwarp();
      const float* wb = wbuf + (ch & 1) * ROTW_CH * 64 + 2 * lane;
      const int cend = min(ROTW_CH, ncol - ch * ROTW_CH);
      if (!pair) {
        for (int u = 0; u < cend; u++) {
          const float2 w = act ? *reinterpret_cast<const float2*>(wb + u * nrow) : make_float2(0.f, 0.f);
          const float2 wx = make_float2(w.x, w.x), wy = make_float2(w.y, w.y);
          const float4* xr = reinterpret_cast<const float4*>(X + (size_t)xrow(ch * ROTW_CH + u) * NCT);
#pragma unroll
          for (int q = 0; q < NCT / 4; q++) {
            const float4 x = xr[q];
            const float2 xl = make_float2(x.x, x.y), xh = make_float2(x.z, x.w);
            a0[2 * q] = __ffma2_rn(wx, xl, a0[2 * q]);
            a0[2 * q + 1] = __ffma2_rn(wx, xh, a0[2 * q + 1]);
            a1[2 * q] = __ffma2_rn(wy, xl, a1[2 * q]);
            a1[2 * q + 1] = __ffma2_rn(wy, xh, a1[2 * q + 1]);
          }
        }
      } else {
        for (int u = 0; u < cend; u += 2) {
          const float2 wr = act ? *reinterpret_cast<const float2*>(wb + u * nrow) : make_float2(0.f, 0.f);
          const float2 wi = act ? *reinterpret_cast<const float2*>(wb + (u + 1) * nrow) : make_float2(0.f, 0.f);
          const int rk = xrow((ch * ROTW_CH + u) >> 1);
          const float4* xre = reinterpret_cast<const float4*>(X + (size_t)rk * NCT);
          const float4* xim = reinterpret_cast<const float4*>(X + (size_t)(rk + 1) * NCT);
          const float2 wrx = make_float2(wr.x, wr.x), wry = make_float2(wr.y, wr.y);
          const float2 wix = make_float2(wi.x, wi.x), wiy = make_float2(wi.y, wi.y);
#pragma unroll
          for (int q = 0; q < NCT / 4; q++) {
            const float4 xr = xre[q], xi = xim[q];
            const float2 rl = make_float2(xr.x, xr.y), rh = make_float2(xr.z, xr.w);
            const float2 il = make_float2(xi.x, xi.y), ih = make_float2(xi.z, xi.w);
            a0[2 * q] = __ffma2_rn(wix, il, __ffma2_rn(wrx, rl, a0[2 * q]));
            a0[2 * q + 1] = __ffma2_rn(wix, ih, __ffma2_rn(wrx, rh, a0[2 * q + 1]));
            a1[2 * q] = __ffma2_rn(wiy, il, __ffma2_rn(wry, rl, a1[2 * q]));
            a1[2 * q + 1] = __ffma2_rn(wiy, ih, __ffma2_rn(wry, rh, a1[2 * q + 1]));
          }
        }
      }
      __syncwarp();  // buffer (ch & 1) is refilled by the fetch of chunk ch + 2
    }
  };
  auto rotate = [&](long long base) {
    for (int n = 0; n <= p; n++) {
      if (owner[n] != warp) continue;
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      float2 a0[NCT / 2], a1[NCT / 2];
#pragma unroll
      for (int c = 0; c < NCT / 2; c++) a0[c] = a1[c] = make_float2(0.0f, 0.0f);
      block(pool + base + rot_block_off(n), bb, bb, false, [&](int k) { return r0 + k; }, a0, a1);
      if (2 * lane < bb) put_rows(r0 + 2 * lane, r0 + 2 * lane + 1, a0, a1);
      __syncwarp();
    }
  };
  rotate(op.fw);
  __syncthreads();
  // shift along z: order block m (rows (n, m), n = m..p), owned like degree block p - m
  for (int m = 0; m <= p; m++) {
    if (owner[p - m] != warp) continue;
    const int bz = 2 * (p - m + 1);
    float2 a0[NCT / 2], a1[NCT / 2];
#pragma unroll
    for (int c = 0; c < NCT / 2; c++) a0[c] = a1[c] = make_float2(0.0f, 0.0f);
    block(pool + op.z + z_block_off(p, m), bz, bz, true,
          [&](int kq) { const int k = m + kq; return 2 * (k * (k + 1) / 2 + m); }, a0, a1);
    if (2 * lane < bz) {
      const int n = m + lane, cc = n * (n + 1) / 2 + m;
      put_rows(2 * cc, 2 * cc + 1, a0, a1);
    }
    __syncwarp();
  }
  __syncthreads();
  rotate(op.bk);
  __syncthreads();
  for (int j = 0; j < NCT; j++) {
    const int col = t.col0 + j;
    if (col >= t.ncols) break;
    const TransPair pr = pairs[t.pair0 + col / C];
    float* dp = dst + ((size_t)pr.dst * C + col % C) * D;
    const float al = (float)pr.alpha;
    for (int r = tid; r < dim; r += ROTW_THREADS) atomicAdd(dp + r, al * X[(size_t)r * NCT + j]);
  }
}

// FP32 translations in the parity-split form (build_split_ops): five factors
// per column, Rz forward (applied while the sources are staged), the re / im
// blocks of Ry forward, of the shift along z and of Ry back (one warp per
// block, in place in shared memory), Rz back (applied to the last blocks'
// results in registers).  Shared layout: per coefficient c one row of the
// task's 16 columns as (re, im) pairs, rows 36 floats apart (the 4-float pad
// keeps the staging and the output conflict-free).  In a block of r rows,
// lane (rp, ch) owns output rows 2 rp, 2 rp + 1 for 16 / CG columns; per
// input row k it reads one float4 of operator (re, im of row 2 rp; re, im of
// row 2 rp + 1; 16 lanes read 256 contiguous bytes) and the (re, im) pairs
// of its columns as shared-memory broadcasts, so that every product is one
// paired FMA (re and im lanes of the pair) with no register moves: CG = 2
// (16 row pairs x 8 columns) for r > 16, CG = 4 (8 row pairs x 4 columns)
// below.  The operator float4 come straight from global memory (L2), PF
// rows ahead in registers; the product loop runs whole groups of PF rows
// with no branch inside (the steps past a block's last row read its zero
// column).  NW warps per CTA, registers sized for MINB CTAs per SM; for
// orders p <= 31.
constexpr int RS_PMAX = 31, RS_NCT = 16, RS_XS = 2 * RS_NCT + 4;
struct RsBlocks {
  int s[RS_PMAX + 3];
};
constexpr RsBlocks make_rs_blocks() {
  RsBlocks b{};
  for (int R = 0; R <= RS_PMAX + 2; R++) b.s[R] = (int)rots_blocks(R);
  return b;
}
__constant__ RsBlocks c_rs_blocks = make_rs_blocks();
// Warp of degree block n at order p (order block p - n of the shift), nw
// warps: a block of r rows costs r steps rounded up to the prefetch depth
// (all its rows are spread over the lanes), a step of the 8-column form
// about twice one of the 4-column form, plus a fixed cost per block; largest
// first onto the least loaded warp.
constexpr RotwOwners make_rs_owners(int nw) {
  RotwOwners o{};
  for (int p = 0; p <= RS_PMAX; p++) {
    int load[16] = {};
    for (int n = p; n >= 0; n--) {
      int best = 0;
      for (int w = 1; w < nw; w++)
        if (load[w] < load[best]) best = w;
      o.o[p][n] = (unsigned char)best;
      const int r = n + 1;
      load[best] += (r + 3) / 4 * 4 * (r > 16 ? 20 : 11) + 60;
    }
  }
  return o;
}
__constant__ RotwOwners c_rs_owners8 = make_rs_owners(8);
__constant__ RotwOwners c_rs_owners12 = make_rs_owners(12);
__host__ __device__ inline size_t rs_cbase_off(int dim) { return sizeof(float) * (size_t)(dim / 2) * RS_XS; }
__host__ __device__ inline size_t rs_smem(int dim) { return rs_cbase_off(dim) + 8 * RS_NCT; }
// float4 f (columns 2f, 2f + 1) of coefficient c in the shared rows
__device__ __forceinline__ float4* rs_x(float* X, int c, int f) { return reinterpret_cast<float4*>(X + c * RS_XS) + f; }

template <int NW, int PF, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB)
k_translate_rot_s(const TransTask* __restrict__ tasks, const TransPair* __restrict__ pairs,
                  const RotSOp* __restrict__ ops, const float* __restrict__ pool, int D, int C,
                  const float* __restrict__ src, float* __restrict__ dst) {
  constexpr int NCT = RS_NCT, XS = RS_XS, NT = NW * 32;
  extern __shared__ __align__(16) unsigned char rs_smem_[];
  const TransTask t = tasks[blockIdx.x];
  const RotSOp op = ops[t.group];
  const int p = op.p, nc = (p + 1) * (p + 2) / 2, dim = 2 * nc;
  const int nblk = c_rs_blocks.s[p + 1];
  const float* g0 = pool + op.base;
  const float4* rzf = reinterpret_cast<const float4*>(g0);
  const float* ryf = g0 + 4 * (p + 1);
  const float* zb = ryf + nblk;
  const float* ryb = zb + nblk;
  const float4* rzb = reinterpret_cast<const float4*>(ryb + nblk);
  float* X = reinterpret_cast<float*>(rs_smem_);                                   // [nc][XS]
  long long* cbase = reinterpret_cast<long long*>(rs_smem_ + rs_cbase_off(dim));  // [NCT]: source columns
  const unsigned char* owner = (NW == 8 ? c_rs_owners8 : c_rs_owners12).o[p];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < NCT) {
    const int col = t.col0 + tid;
    long long b = -1;
    if (col < t.ncols) {
      const TransPair pr = pairs[t.pair0 + col / C];
      b = ((long long)pr.src * C + col % C) * D;
    }
    cbase[tid] = b;
  }
  __syncthreads();
  // stage the sources with Rz forward: thread (coefficient, 4 columns)
  for (int q = tid; q < nc * (NCT / 4); q += NT) {
    const int c = q % nc, cg = q / nc;
    int n, m;
    coef_nm(c, n, m);
    const float4 R = __ldg(rzf + m);
    float2 v[4];
#pragma unroll
    for (int g = 0; g < 4; g++) {
      const long long b = cbase[cg * 4 + g];
      const float2 s = b >= 0 ? __ldg(reinterpret_cast<const float2*>(src + b + 2 * c)) : make_float2(0.f, 0.f);
      v[g] = make_float2(R.x * s.x + R.y * s.y, R.z * s.x + R.w * s.y);
    }
    *rs_x(X, c, 2 * cg) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    *rs_x(X, c, 2 * cg + 1) = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
  }
  __syncthreads();
  // one block of r rows (operator columns at blk, h float4 each, then a
  // zero column); row k of the block is coefficient c(k) = c0 + k (Ry:
  // dc = 0) or c0 + k (i + 1) + k (k - 1) / 2 (the shift's order block i:
  // c(k + 1) - c(k) = i + k + 1, dc = 1); the results go back to the same
  // coefficients, through rz (4 per order, indexed by the row) when given.
  // Lanes past the block's rows read the last row pair's operator (no
  // divergence in the product loop) and write nothing.
  auto block = [&](auto cgtag, const float* blk, int r, int c0, int i, int dc, const float4* rz) {
    constexpr int CG = decltype(cgtag)::value, RP = 32 / CG, COLS = NCT / CG, NF = COLS / 2;
    const int h = (r + 1) / 2, rp = lane % RP, ch = lane / RP;
    const bool act = rp < h;
    const float4* opp = reinterpret_cast<const float4*>(blk) + min(rp, h - 1);
    float2 a0[COLS], a1[COLS];  // (re, im) of rows 2 rp, 2 rp + 1 per column
#pragma unroll
    for (int v = 0; v < COLS; v++) a0[v] = a1[v] = make_float2(0.f, 0.f);
    // shared position of row k: xo (floats from X), advanced by xs per row,
    // xs growing by dxs (the shift's rows lie further apart as n grows);
    // the steps past the last row read the zero operator column r and the
    // last row
    int xo = c0 * XS + ch * 2 * COLS;
    int xs = dc ? (i + 1) * XS : XS;
    const int dxs = dc ? XS : 0;
    const int xlast = xo + (dc ? (r - 1) * (i + 1) + (r - 1) * (r - 2) / 2 : r - 1) * XS;
    // operator rows k .. k + PF - 1 in flight
    float4 oq[PF];
#pragma unroll
    for (int j = 0; j < PF; j++) oq[j] = __ldg(opp + min(j, r) * h);
    const int nit = (r + PF - 1) / PF;
    for (int it = 0, k = PF; it < nit; it++) {
#pragma unroll
      for (int j = 0; j < PF; j++, k++) {
        const float4 o = oq[j];
        oq[j] = __ldg(opp + min(k, r) * h);
        const float2 w0 = make_float2(o.x, o.y), w1 = make_float2(o.z, o.w);
        const float4* xq = reinterpret_cast<const float4*>(X + min(xo, xlast));
        xo += xs;
        xs += dxs;
#pragma unroll
        for (int f = 0; f < NF; f++) {
          const float4 x = xq[f];
          const float2 xa = make_float2(x.x, x.y), xb = make_float2(x.z, x.w);
          a0[2 * f] = __ffma2_rn(w0, xa, a0[2 * f]);
          a0[2 * f + 1] = __ffma2_rn(w0, xb, a0[2 * f + 1]);
          a1[2 * f] = __ffma2_rn(w1, xa, a1[2 * f]);
          a1[2 * f + 1] = __ffma2_rn(w1, xb, a1[2 * f + 1]);
        }
      }
    }
    __syncwarp();  // every lane's reads of the block's rows are done
    auto put = [&](int k, const float2* a) {
      const int c = c0 + (dc ? k * (i + 1) + k * (k - 1) / 2 : k);
      float2 o[COLS];
      if (rz) {
        const float4 R = __ldg(rz + k);
#pragma unroll
        for (int e = 0; e < COLS; e++) o[e] = make_float2(R.x * a[e].x + R.y * a[e].y, R.z * a[e].x + R.w * a[e].y);
      } else {
#pragma unroll
        for (int e = 0; e < COLS; e++) o[e] = a[e];
      }
#pragma unroll
      for (int f = 0; f < NF; f++) *rs_x(X, c, ch * NF + f) = make_float4(o[2 * f].x, o[2 * f].y, o[2 * f + 1].x, o[2 * f + 1].y);
    };
    if (act) {
      put(2 * rp, a0);
      if (2 * rp + 1 < r) put(2 * rp + 1, a1);
    }
    __syncwarp();
  };
  // the three factors: degree blocks n of Ry forward, order blocks m of the
  // shift (owned like degree block p - m), degree blocks of Ry back
  for (int st = 0; st < 3; st++) {
    for (int i = 0; i <= p; i++) {
      if (owner[st == 1 ? p - i : i] != warp) continue;
      const int r = st == 1 ? p - i + 1 : i + 1;
      const float* blk = st == 1 ? zb + nblk - c_rs_blocks.s[p + 1 - i] : (st == 0 ? ryf : ryb) + c_rs_blocks.s[i];
      // first coefficient of the block: (i, i) for the shift's order i, (i, 0) for degree i
      const int c0 = i * (i + 1) / 2 + (st == 1 ? i : 0);
      const float4* rz = st == 2 ? rzb : nullptr;
      if (r > 16)
        block(std::integral_constant<int, 2>{}, blk, r, c0, i, st == 1, rz);
      else
        block(std::integral_constant<int, 4>{}, blk, r, c0, i, st == 1, rz);
    }
    __syncthreads();
  }
  for (int j = 0; j < NCT; j++) {
    const int col = t.col0 + j;
    if (col >= t.ncols) break;
    const TransPair pr = pairs[t.pair0 + col / C];
    float* dp = dst + ((size_t)pr.dst * C + col % C) * D;
    const float al = (float)pr.alpha;
    for (int r = tid; r < dim; r += NT) {
      const float* x = reinterpret_cast<const float*>(rs_x(X, r >> 1, j >> 1));
      atomicAdd(dp + r, al * x[2 * (j & 1) + (r & 1)]);
    }
  }
}

bool rot_split_ok(int maxdim) { return maxdim <= (RS_PMAX + 1) * (RS_PMAX + 2); }

// Columns per CTA of the split kernel.
int rot_split_cols() { return RS_NCT; }

// Variants of the split kernel (warps, operator rows ahead, CTAs per SM the
// registers are sized for): 1 (12, 2, 2), 2 (8, 4, 2), 3 (8, 2, 3), 4 (8, 6,
// 2), 5 (8, 8, 2); <= 0 takes ELFMM3D_ROTS_VARIANT, default 3.
void launch_translate_rot_split(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                                const RotSOp* ops, const float* pool, int D, int C, int maxdim, const float* src,
                                float* dst, int variant) {
  if (ntask <= 0) return;
  if (!rot_split_ok(maxdim)) throw CudaError{(int)cudaErrorInvalidValue};
  static const int v_env = [] {
    const char* e = getenv("ELFMM3D_ROTS_VARIANT");
    const int v = e ? atoi(e) : 3;
    return (v >= 1 && v <= 5) ? v : 3;
  }();
  const int v = variant > 0 ? variant : v_env;
  if (v < 1 || v > 5) throw CudaError{(int)cudaErrorInvalidValue};
  const size_t smem = rs_smem(maxdim);
  auto go = [&](auto kern, int nw) {
    EFMM_CUDA_TRY(smem_raise(kern, (int)smem));
    kern<<<ntask, nw * 32, smem, st>>>(tasks, pairs, ops, pool, D, C, src, dst);
  };
  if (v == 1)
    go(k_translate_rot_s<12, 2, 2>, 12);
  else if (v == 2)
    go(k_translate_rot_s<8, 4, 2>, 8);
  else if (v == 3)
    go(k_translate_rot_s<8, 2, 3>, 8);
  else if (v == 4)
    go(k_translate_rot_s<8, 6, 2>, 8);
  else
    go(k_translate_rot_s<8, 8, 2>, 8);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

// M2L of the half-space kernel U in the parity-split form (build_usplit_ops):
// a task is one output tile of 64 coefficient rows x 128 columns of a group
// (columns: the concatenated columns of the group's pairs, as k_translate),
// both parts at once: the B tile loader reads each source coefficient's re
// and im words once and keeps both parts of its Rz in rotation, the CTA
// accumulates the re block's and the im block's products side by side, and
// the epilogue rotates each (re, im) result pair by Rz out and adds it into
// the destination with one atomic per real row.  256 threads, 4 x 8 outputs
// of each part per thread, K tiles of 16 double-buffered in shared memory;
// half the multiply-adds of the dense operator.
constexpr int US_R = 64, US_C = 128, US_K = 16, US_PMAX = 63;
struct UsMof {
  unsigned char m[(US_PMAX + 1) * (US_PMAX + 2) / 2];
};
constexpr UsMof make_us_mof() {
  UsMof t{};
  for (int n = 0; n <= US_PMAX; n++)
    for (int m = 0; m <= n; m++) t.m[n * (n + 1) / 2 + m] = (unsigned char)m;
  return t;
}
__constant__ UsMof c_us_mof = make_us_mof();
constexpr int US_SMEM = (int)sizeof(float) * 2 * US_K * (2 * US_R + 2 * US_C);

__global__ void __launch_bounds__(256, 2)
k_translate_us(const TransTask* __restrict__ tasks, const TransPair* __restrict__ pairs,
               const USOp* __restrict__ ops, const float* __restrict__ pool, int D, int C,
               const float* __restrict__ src, float* __restrict__ dst) {
  extern __shared__ __align__(16) float us_smem[];
  float* Ar = us_smem;                   // [2][US_K][US_R]
  float* Ai = Ar + 2 * US_K * US_R;      // [2][US_K][US_R]
  float* Br = Ai + 2 * US_K * US_R;      // [2][US_K][US_C]
  float* Bi = Br + 2 * US_K * US_C;      // [2][US_K][US_C]
  const TransTask t = tasks[blockIdx.x];
  const int r0 = t.row0;
  const USOp op = ops[t.group];
  const int nc = (op.p + 1) * (op.p + 2) / 2, ld = op.ld;
  const float4* rzi = reinterpret_cast<const float4*>(pool + op.rzi);
  const float4* rzo = reinterpret_cast<const float4*>(pool + op.rzo);
  const int tid = threadIdx.x;
  // loader roles: A row (tid >> 2), 4 k (tid & 3); B column (tid & 127), k half (tid >> 7)
  const int arow = tid >> 2, akq = (tid & 3) * 4;
  const bool arow_ok = r0 + arow < nc;
  const float* Apr = pool + op.re + (size_t)(arow_ok ? r0 + arow : 0) * ld;
  const float* Api = pool + op.im + (size_t)(arow_ok ? r0 + arow : 0) * ld;
  const int bcol = tid & 127, bkh = (tid >> 7) * 8;
  const float* Bp = nullptr;
  {
    const int col = t.col0 + bcol;
    if (col < t.ncols) {
      const TransPair pr = pairs[t.pair0 + col / C];
      Bp = src + ((size_t)pr.src * C + (col % C)) * D;
    }
  }
  float rar[4], rai[4], rbr[8], rbi[8];
  auto load = [&](int k0) {
    const int ka = k0 + akq, kb = k0 + bkh;
    if (arow_ok && ka + 4 <= nc) {
      const float4 u = *reinterpret_cast<const float4*>(Apr + ka);
      const float4 v = *reinterpret_cast<const float4*>(Api + ka);
      rar[0] = u.x; rar[1] = u.y; rar[2] = u.z; rar[3] = u.w;
      rai[0] = v.x; rai[1] = v.y; rai[2] = v.z; rai[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const bool ok = arow_ok && ka + i < nc;
        rar[i] = ok ? Apr[ka + i] : 0.0f;
        rai[i] = ok ? Api[ka + i] : 0.0f;
      }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = kb + i;
      float vr = 0.0f, vi = 0.0f;
      if (Bp && c < nc) {
        const float2 x = *reinterpret_cast<const float2*>(Bp + 2 * c);
        const float4 R = __ldg(rzi + c_us_mof.m[c]);
        vr = R.x * x.x + R.y * x.y;
        vi = R.z * x.x + R.w * x.y;
      }
      rbr[i] = vr;
      rbi[i] = vi;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      Ar[(buf * US_K + akq + i) * US_R + arow] = rar[i];
      Ai[(buf * US_K + akq + i) * US_R + arow] = rai[i];
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      Br[(buf * US_K + bkh + i) * US_C + bcol] = rbr[i];
      Bi[(buf * US_K + bkh + i) * US_C + bcol] = rbi[i];
    }
  };
  const int tx = tid & 15, ty = tid >> 4;
  float cr[4][8], ci[4][8];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) cr[i][j] = ci[i][j] = 0.0f;
  const int nk = (nc + US_K - 1) / US_K;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; kt++) {
    const int cur = kt & 1;
    if (kt + 1 < nk) load((kt + 1) * US_K);
#pragma unroll
    for (int kk = 0; kk < US_K; kk++) {
      const float4 ar = *reinterpret_cast<const float4*>(&Ar[(cur * US_K + kk) * US_R + ty * 4]);
      const float4 ai = *reinterpret_cast<const float4*>(&Ai[(cur * US_K + kk) * US_R + ty * 4]);
      const float a_r[4] = {ar.x, ar.y, ar.z, ar.w}, a_i[4] = {ai.x, ai.y, ai.z, ai.w};
      float b_r[8], b_i[8];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float2 u = *reinterpret_cast<const float2*>(&Br[(cur * US_K + kk) * US_C + 32 * j + 2 * tx]);
        const float2 v = *reinterpret_cast<const float2*>(&Bi[(cur * US_K + kk) * US_C + 32 * j + 2 * tx]);
        b_r[2 * j] = u.x;
        b_r[2 * j + 1] = u.y;
        b_i[2 * j] = v.x;
        b_i[2 * j + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          cr[i][j] += a_r[i] * b_r[j];
          ci[i][j] += a_i[i] * b_i[j];
        }
    }
    if (kt + 1 < nk) store(cur ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int col = t.col0 + 32 * (j >> 1) + 2 * tx + (j & 1);
    if (col >= t.ncols) continue;
    const TransPair pr = pairs[t.pair0 + col / C];
    float* dp = dst + ((size_t)pr.dst * C + (col % C)) * D;
    const float al = (float)pr.alpha;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int r = r0 + ty * 4 + i;
      if (r < nc) {
        const float4 R = __ldg(rzo + c_us_mof.m[r]);
        atomicAdd(dp + 2 * r, al * (R.x * cr[i][j] + R.y * ci[i][j]));
        atomicAdd(dp + 2 * r + 1, al * (R.z * cr[i][j] + R.w * ci[i][j]));
      }
    }
  }
}

void launch_translate_us(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs, const USOp* ops,
                         const float* pool, int D, int C, const float* src, float* dst) {
  if (ntask <= 0) return;
  EFMM_CUDA_TRY(smem_raise(k_translate_us, US_SMEM));
  k_translate_us<<<ntask, 256, US_SMEM, st>>>(tasks, pairs, ops, pool, D, C, src, dst);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

// The warp-block kernel for launches of orders pmin..31 (smaller orders
// have fewer blocks than warps: the coefficient-tile kernel serves them).
bool rot_warp_blocks_ok(int maxdim) {
  static const int pmin = [] {
    const char* e = getenv("ELFMM3D_ROTW_PMIN");
    return e ? atoi(e) : 20;
  }();
  return maxdim <= (ROTW_PMAX + 1) * (ROTW_PMAX + 2) && maxdim >= (pmin + 1) * (pmin + 2);
}

int rot_cols_per_cta(int maxdim, int elem_bytes) {
  (void)maxdim;
  return elem_bytes == 4 ? 16 : 8;
}

template <class T>
void launch_translate_rot(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                          const RotOp* ops, const T* pool, int D, int C, int maxdim, const T* src, T* dst) {
  if (ntask <= 0) return;
  static const bool warp_blocks = [] {
    const char* e = getenv("ELFMM3D_ROT");
    return !(e && strcmp(e, "tiles") == 0);
  }();
  if constexpr (sizeof(T) == 4) {
    if (warp_blocks && rot_warp_blocks_ok(maxdim)) {
      const size_t smem = rotw_smem(maxdim);
      EFMM_CUDA_TRY(smem_raise(k_translate_rot_w, (int)smem));
      k_translate_rot_w<<<ntask, ROTW_THREADS, smem, st>>>(tasks, pairs, ops, reinterpret_cast<const float*>(pool),
                                                             D, C, reinterpret_cast<const float*>(src),
                                                             reinterpret_cast<float*>(dst));
      count_launch();
      EFMM_CUDA_TRY(cudaGetLastError());
      return;
    }
  }
  constexpr int NCT = sizeof(T) == 4 ? 16 : 8;
  const size_t smem = sizeof(T) * 2 * (size_t)maxdim * NCT;
  if (smem > 227 * 1024) throw CudaError{(int)cudaErrorInvalidValue};
  auto kern = k_translate_rot<T, NCT>;
  EFMM_CUDA_TRY(smem_raise(kern, (int)smem));
  kern<<<ntask, ROT_THREADS, smem, st>>>(tasks, pairs, ops, pool, D, C, src, dst); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}
template void launch_translate_rot<double>(cudaStream_t, int, const TransTask*, const TransPair*, const RotOp*,
                                           const double*, int, int, int, const double*, double*);
template void launch_translate_rot<float>(cudaStream_t, int, const TransTask*, const TransPair*, const RotOp*,
                                          const float*, int, int, int, const float*, float*);

}  // namespace efmm

// CPU self-check of the factored operators (no device needed): largest
// relative difference to the dense operators over every `stride`-th group of
// the M2L offsets (|max| 2..3 in [-3,3]^3) and the 8 M2M and 8 L2L shifts at
// order p and tolerance eps.  Returns the number of groups built.
extern "C" int efmm_factored_selfcheck(int p, double eps, int stride, double* worst) {
  using namespace efmm;
  std::vector<int> kinds, orders;
  std::vector<double> offs;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        if (std::max(std::abs(i), std::max(std::abs(j), std::abs(k))) < 2) continue;
        kinds.push_back(0);
        orders.push_back(std::min(p, eps > 0 ? m2l_order(eps, i, j, k) : p));
        offs.insert(offs.end(), {(double)i, (double)j, (double)k});
      }
  for (int kind = 1; kind <= 2; kind++)
    for (int dg = 0; dg < 8; dg++) {
      kinds.push_back(kind);
      orders.push_back(p);
      offs.insert(offs.end(), {(dg & 1) ? 0.25 : -0.25, ((dg >> 1) & 1) ? 0.25 : -0.25,
                               ((dg >> 2) & 1) ? 0.25 : -0.25});
    }
  std::vector<RotOp> ops;
  std::vector<double> pool;
  build_factored_ops(p, kinds, orders, offs, ops, pool);
  *worst = check_factored_ops(kinds, orders, offs, ops, pool, stride);
  return (int)kinds.size();
}

namespace efmm {
namespace {
// The packed FP32 pool of one group applied on the host exactly as the
// device kernel reads it (normalised basis): layout check without a device.
void apply_split_packed(const float* g, int p, const std::vector<double>& v, std::vector<double>& y) {
  const int nc = ncoef(p), dim = 2 * nc;
  const long long nb = rots_blocks(p + 1);
  const float* rzf = g;
  const float* ryf = g + 4 * (p + 1);
  const float* zb = ryf + nb;
  const float* ryb = zb + nb;
  const float* rzb = ryb + nb;
  std::vector<double> x(v);
  auto rz = [&](const float* R) {
    for (int n = 0; n <= p; n++)
      for (int m = 0; m <= n; m++) {
        const int c = 2 * cidx(n, m);
        const double re = x[c], im = x[c + 1];
        x[c] = R[4 * m] * re + R[4 * m + 1] * im;
        x[c + 1] = R[4 * m + 2] * re + R[4 * m + 3] * im;
      }
  };
  auto blk = [&](const float* B, int r, auto row) {
    const int h = (r + 1) / 2;
    std::vector<double> o(2 * r, 0.0);
    for (int k = 0; k < r; k++)
      for (int i = 0; i < r; i++) {
        const float* q = B + ((size_t)k * h + i / 2) * 4 + 2 * (i & 1);
        o[2 * i] += q[0] * x[row(k)];
        o[2 * i + 1] += q[1] * x[row(k) + 1];
      }
    for (int i = 0; i < r; i++) {
      x[row(i)] = o[2 * i];
      x[row(i) + 1] = o[2 * i + 1];
    }
  };
  rz(rzf);
  for (int n = 0; n <= p; n++) blk(ryf + rots_blocks(n), n + 1, [&](int k) { return n * (n + 1) + 2 * k; });
  for (int m = 0; m <= p; m++)
    blk(zb + nb - rots_blocks(p + 1 - m), p - m + 1, [&](int k) { return (m + k) * (m + k + 1) + 2 * m; });
  for (int n = 0; n <= p; n++) blk(ryb + rots_blocks(n), n + 1, [&](int k) { return n * (n + 1) + 2 * k; });
  rz(rzb);
  y.assign(x.begin(), x.begin() + dim);
}
}  // namespace
}  // namespace efmm

// CPU self-check of the parity-split factors (no device needed), over the
// same groups as efmm_factored_selfcheck: worst[0] the split factors in
// double against the dense operators, worst[1] the packed FP32 device pool
// applied as the kernel reads it, worst[2] the largest coupling the split
// drops (re <-> im terms of Ry and the shift, off-order terms of Rz).
extern "C" int efmm_split_selfcheck(int p, double eps, int stride, double* worst) {
  using namespace efmm;
  std::vector<int> kinds, orders;
  std::vector<double> offs;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        if (std::max(std::abs(i), std::max(std::abs(j), std::abs(k))) < 2) continue;
        kinds.push_back(0);
        orders.push_back(std::min(p, eps > 0 ? m2l_order(eps, i, j, k) : p));
        offs.insert(offs.end(), {(double)i, (double)j, (double)k});
      }
  for (int kind = 1; kind <= 2; kind++)
    for (int dg = 0; dg < 8; dg++) {
      kinds.push_back(kind);
      orders.push_back(p);
      offs.insert(offs.end(), {(dg & 1) ? 0.25 : -0.25, ((dg >> 1) & 1) ? 0.25 : -0.25,
                               ((dg >> 2) & 1) ? 0.25 : -0.25});
    }
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<RotSOp> sops;
  std::vector<float> spool;
  build_split_ops(kinds, orders, offs, w, sops, spool);
  Fitter F;
  F.init(p);
  worst[0] = worst[1] = worst[2] = 0;
  std::mt19937_64 rng(11);
  std::normal_distribution<double> N01;
  for (int g = 0; g < (int)kinds.size(); g += std::max(stride, 1)) {
    const int kind = kinds[g], pg = orders[g], nc = ncoef(pg), dim = 2 * nc;
    const double* d = &offs[3 * g];
    SplitHost S;
    build_split_host(kind, pg, d, F, S);
    worst[2] = std::max(worst[2], S.cross);
    std::vector<cplx> tab(ncoef(2 * pg + 1));
    if (kind == 0)
      irregular_harmonics(2 * pg, d[0], d[1], d[2], tab.data());
    else
      regular_harmonics(pg, d[0], d[1], d[2], tab.data());
    const bool in_local = kind == 2, out_local = kind != 1;
    std::vector<double> v(dim), a(dim, 0.0), vn(dim), y, yn;
    for (int q = 0; q < dim; q++) v[q] = N01(rng) * (in_local ? w[q] : 1.0 / w[q]);
    for (int n = 0; n <= pg; n++) v[2 * cidx(n, 0) + 1] = 0.0;
    for (int r = 0; r < nc; r++)
      for (int c = 0; c < nc; c++) {
        double rr, ri, ir, ii;
        op_entry(kind, tab.data(), r, c, &rr, &ri, &ir, &ii);
        a[2 * r] += rr * v[2 * c] + ri * v[2 * c + 1];
        a[2 * r + 1] += ir * v[2 * c] + ii * v[2 * c + 1];
      }
    apply_split_host(S, v, y);
    for (int q = 0; q < dim; q++) vn[q] = v[q] * (in_local ? 1.0 / w[q] : w[q]);
    apply_split_packed(&spool[sops[g].base], pg, vn, yn);
    double num0 = 0, num1 = 0, den = 0;
    for (int n = 0; n <= pg; n++)
      for (int m = 0; m <= n; m++)
        for (int part = 0; part < 2; part++) {
          if (m == 0 && part == 1) continue;
          const int q = 2 * cidx(n, m) + part;
          const double sc = out_local ? 1.0 / w[q] : w[q];
          const double y1 = yn[q] / sc;
          num0 += (a[q] - y[q]) * (a[q] - y[q]) * sc * sc;
          num1 += (a[q] - y1) * (a[q] - y1) * sc * sc;
          den += a[q] * a[q] * sc * sc;
        }
    worst[0] = std::max(worst[0], std::sqrt(num0 / std::max(den, 1e-300)));
    worst[1] = std::max(worst[1], std::sqrt(num1 / std::max(den, 1e-300)));
  }
  return (int)kinds.size();
}

// Device run of the FP32 translation kernels on four groups of order p (an
// M2L offset, one along -z, an M2M and an L2L shift), npair box pairs each
// with C columns per box (random normalised sources, pair factors alpha, one
// destination box per group), in one launch.  engine 0: the parity-split
// kernel (k_translate_rot_s, default variant); 1: the full-block kernels
// (k_translate_rot_w / k_translate_rot, as launch_translate_rot<float> picks
// them); 2..6: the split kernel's variants 1..5.  reps > 0
// then times reps more launches (mean ms in *ms).  With rel: the relative l2
// error of the destinations of the first launch against the split factors
// of the same FP32 pool applied in FP64 on the host.
static int rot_split_device_run(int p, int C, int npair, unsigned seed, int engine, int reps, double* rel,
                                double* ms) {
  using namespace efmm;
  if (p < 1 || p > 31 || C < 1 || npair < 1 || (long long)C * npair > (1 << 20) || engine < 0 || engine > 6)
    return 16;
  const int NG = 4;
  std::vector<int> kinds = {0, 0, 1, 2}, orders(NG, p);
  std::vector<double> offs = {2, -1, 3, 0, 0, -2, 0.25, 0.25, -0.25, -0.25, 0.25, 0.25};
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<RotSOp> sops;
  std::vector<float> spool;
  build_split_ops(kinds, orders, offs, w, sops, spool);
  std::vector<RotOp> rops;
  std::vector<double> pool;
  std::vector<float> poolf;
  if (engine == 1) {
    build_factored_ops(p, kinds, orders, offs, rops, pool);
    normalise_factored_ops(kinds, rops, pool, w, poolf);
    std::vector<double> tmp(poolf.begin(), poolf.end());
    column_major_factored(rops, tmp);
    for (size_t i = 0; i < tmp.size(); i++) poolf[i] = (float)tmp[i];
  }
  const int D = 2 * ncoef(p), dim = D;
  const int nsrc = NG * npair, nbox = nsrc + NG;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> U(-1.f, 1.f);
  std::vector<float> hsrc((size_t)nbox * C * D, 0.f), hdst((size_t)nbox * C * D, 0.f);
  for (int b = 0; b < nsrc; b++)
    for (int c = 0; c < C; c++)
      for (int q = 0; q < D; q++) {
        const bool m0im = (q & 1) && q / 2 == cidx((int)((std::sqrt(8.0 * (q / 2) + 1) - 1) / 2), 0);
        hsrc[((size_t)b * C + c) * D + q] = m0im ? 0.f : U(rng);
      }
  std::vector<TransPair> hp;
  std::vector<TransTask> tasks;
  for (int g = 0; g < NG; g++) {
    for (int k = 0; k < npair; k++) hp.push_back({g * npair + k, nsrc + g, 0.5 + 0.25 * k});
    const int ncols = npair * C;
    for (int c0 = 0; c0 < ncols; c0 += RS_NCT) tasks.push_back({g, 0, g * npair, ncols, c0});
  }
  float *dsrc = nullptr, *ddst = nullptr, *dpool = nullptr;
  TransPair* dp = nullptr;
  TransTask* dtask = nullptr;
  RotSOp* dsops = nullptr;
  RotOp* drops = nullptr;
  auto release = [&]() {
    cudaFree(dsrc); cudaFree(ddst); cudaFree(dpool); cudaFree(dp); cudaFree(dtask); cudaFree(dsops); cudaFree(drops);
  };
  const size_t pbytes = 4 * (engine != 1 ? spool.size() : poolf.size());
  if (cudaMalloc(&dsrc, hsrc.size() * 4) || cudaMalloc(&ddst, hdst.size() * 4) || cudaMalloc(&dpool, pbytes) ||
      cudaMalloc(&dp, hp.size() * sizeof(TransPair)) || cudaMalloc(&dtask, tasks.size() * sizeof(TransTask)) ||
      cudaMalloc(&dsops, sops.size() * sizeof(RotSOp)) || cudaMalloc(&drops, NG * sizeof(RotOp))) {
    release();
    return 256;
  }
  cudaMemcpy(dsrc, hsrc.data(), hsrc.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(ddst, hdst.data(), hdst.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dpool, engine != 1 ? spool.data() : poolf.data(), pbytes, cudaMemcpyHostToDevice);
  cudaMemcpy(dp, hp.data(), hp.size() * sizeof(TransPair), cudaMemcpyHostToDevice);
  cudaMemcpy(dtask, tasks.data(), tasks.size() * sizeof(TransTask), cudaMemcpyHostToDevice);
  cudaMemcpy(dsops, sops.data(), sops.size() * sizeof(RotSOp), cudaMemcpyHostToDevice);
  if (engine == 1) cudaMemcpy(drops, rops.data(), NG * sizeof(RotOp), cudaMemcpyHostToDevice);
  auto launch = [&]() {
    if (engine != 1)
      launch_translate_rot_split(0, (int)tasks.size(), dtask, dp, dsops, dpool, D, C, dim, dsrc, ddst,
                                 engine == 0 ? 0 : engine - 1);
    else
      launch_translate_rot<float>(0, (int)tasks.size(), dtask, dp, drops, dpool, D, C, dim, dsrc, ddst);
  };
  try {
    launch();
  } catch (const CudaError&) {
    release();
    return 256;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    release();
    return 256;
  }
  cudaMemcpy(hdst.data(), ddst, hdst.size() * 4, cudaMemcpyDeviceToHost);
  if (reps > 0 && ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    try {
      for (int r = 0; r < reps; r++) launch();
    } catch (const CudaError&) {
      release();
      return 256;
    }
    cudaEventRecord(e1, 0);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      release();
      return 256;
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  release();
  if (!rel) return 0;
  double num = 0, den = 0;
  for (int g = 0; g < NG; g++)
    for (int c = 0; c < C; c++) {
      std::vector<double> ref(dim, 0.0), v(dim), y;
      for (int k = 0; k < npair; k++) {
        const float* s = &hsrc[((size_t)(g * npair + k) * C + c) * D];
        for (int q = 0; q < dim; q++) v[q] = s[q];
        apply_split_packed(&spool[sops[g].base], p, v, y);
        for (int q = 0; q < dim; q++) ref[q] += (0.5 + 0.25 * k) * y[q];
      }
      const float* got = &hdst[((size_t)(nsrc + g) * C + c) * D];
      for (int n = 0; n <= p; n++)
        for (int m = 0; m <= n; m++)
          for (int part = 0; part < 2; part++) {
            if (m == 0 && part == 1) continue;
            const int q = 2 * cidx(n, m) + part;
            num += (got[q] - ref[q]) * (got[q] - ref[q]);
            den += ref[q] * ref[q];
          }
    }
  *rel = std::sqrt(num / std::max(den, 1e-300));
  return 0;
}

extern "C" int efmm_rot_split_selfcheck_device(int p, int C, int npair, unsigned seed, int engine, double* rel) {
  if (!rel) return 16;
  return rot_split_device_run(p, C, npair, seed, engine, 0, rel, nullptr);
}

// Mean ms of reps launches of the kernel of `engine` on the same inputs.
extern "C" int efmm_rot_split_bench(int p, int C, int npair, int engine, int reps, double* ms) {
  if (reps < 1 || !ms) return 16;
  return rot_split_device_run(p, C, npair, 1, engine, reps, nullptr, ms);
}

// CPU self-check of the parity-split U-kernel M2L (no device needed), over
// every stride-th of the U groups (offsets with max |i|, |j|, |k| in 2..3,
// dz >= 0) at order p and tolerance eps: worst[0] the split in double (Rz
// fitted, blocks of T(d0)) against T(d), worst[1] the packed FP32 pool
// applied as the kernel reads it, worst[2] the re / im coupling dropped.
extern "C" int efmm_usplit_selfcheck(int p, double eps, int stride, double* worst) {
  using namespace efmm;
  if (p < 1 || p > 40 || !worst) return -1;
  std::vector<int> orders;
  std::vector<double> offs;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = 0; k <= 3; k++) {
        if (std::max(std::abs(i), std::max(std::abs(j), std::abs(k))) < 2) continue;
        orders.push_back(std::min(p, eps > 0 ? m2l_order(eps, i, j, k) : p));
        offs.insert(offs.end(), {(double)i, (double)j, (double)k});
      }
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<USOp> ops;
  std::vector<float> pool;
  build_usplit_ops(orders, offs, w, ops, pool, &worst[2]);
  Fitter F;
  F.init(p);
  worst[0] = worst[1] = 0;
  std::mt19937_64 rng(13);
  std::normal_distribution<double> N01;
  for (int g = 0; g < (int)orders.size(); g += std::max(stride, 1)) {
    const int pg = orders[g], nc = ncoef(pg), dim = 2 * nc;
    const double* d = &offs[3 * g];
    std::vector<double> T, T0;
    u_dense(pg, d, T);
    const double d0[3] = {std::sqrt(d[0] * d[0] + d[1] * d[1]), 0.0, d[2]};
    u_dense(pg, d0, T0);
    const double ph = (d[0] == 0.0 && d[1] == 0.0) ? 0.0 : std::atan2(d[1], d[0]);
    double Qz[9], Qzt[9];
    rot_z(-ph, Qz);
    rot_z(ph, Qzt);
    std::vector<double> full(rot_size(pg)), ri, ro;
    F.rotation(0, pg, Qz, full.data());
    split_rz(full, pg, ri);
    F.rotation(1, pg, Qzt, full.data());
    split_rz(full, pg, ro);
    std::vector<int> mof(nc);
    for (int n = 0; n <= pg; n++)
      for (int m = 0; m <= n; m++) mof[cidx(n, m)] = m;
    // a random multipole expansion of a real field, O(1) in the normalised basis
    std::vector<double> v(dim), a(dim, 0.0), x(dim), y(dim, 0.0), xn(dim), yn(dim, 0.0);
    for (int q = 0; q < dim; q++) v[q] = N01(rng) / w[q];
    for (int c = 0; c < nc; c++)
      if (mof[c] == 0) v[2 * c + 1] = 0.0;
    for (int r = 0; r < dim; r++)
      for (int c = 0; c < dim; c++) a[r] += T[(size_t)r * dim + c] * v[c];
    // double: y = Rz_out T0 Rz_in v (re / im blocks of T0 only)
    for (int c = 0; c < nc; c++) {
      const double* R = &ri[4 * mof[c]];
      x[2 * c] = R[0] * v[2 * c] + R[1] * v[2 * c + 1];
      x[2 * c + 1] = R[2] * v[2 * c] + R[3] * v[2 * c + 1];
    }
    std::vector<double> t(dim, 0.0);
    for (int r = 0; r < nc; r++)
      for (int c = 0; c < nc; c++) {
        t[2 * r] += T0[(size_t)(2 * r) * dim + 2 * c] * x[2 * c];
        t[2 * r + 1] += T0[(size_t)(2 * r + 1) * dim + 2 * c + 1] * x[2 * c + 1];
      }
    for (int r = 0; r < nc; r++) {
      const double* R = &ro[4 * mof[r]];
      y[2 * r] = R[0] * t[2 * r] + R[1] * t[2 * r + 1];
      y[2 * r + 1] = R[2] * t[2 * r] + R[3] * t[2 * r + 1];
    }
    // the packed FP32 pool as the kernel reads it (normalised basis)
    const USOp& o = ops[g];
    for (int c = 0; c < nc; c++) {
      const float* R = &pool[o.rzi + 4 * mof[c]];
      const double re = v[2 * c] * w[2 * c], im = v[2 * c + 1] * w[2 * c + 1];
      xn[2 * c] = R[0] * re + R[1] * im;
      xn[2 * c + 1] = R[2] * re + R[3] * im;
    }
    for (int r = 0; r < nc; r++) {
      double sr = 0, si = 0;
      for (int c = 0; c < nc; c++) {
        sr += pool[o.re + (size_t)r * o.ld + c] * xn[2 * c];
        si += pool[o.im + (size_t)r * o.ld + c] * xn[2 * c + 1];
      }
      const float* R = &pool[o.rzo + 4 * mof[r]];
      yn[2 * r] = (R[0] * sr + R[1] * si) * w[2 * r];
      yn[2 * r + 1] = (R[2] * sr + R[3] * si) * w[2 * r + 1];
    }
    double num0 = 0, num1 = 0, den = 0;
    for (int c = 0; c < nc; c++)
      for (int part = 0; part < 2; part++) {
        if (mof[c] == 0 && part == 1) continue;
        const int q = 2 * c + part;
        const double sc = 1.0 / w[q];  // the normalised local basis
        num0 += (a[q] - y[q]) * (a[q] - y[q]) * sc * sc;
        num1 += (a[q] - yn[q]) * (a[q] - yn[q]) * sc * sc;
        den += a[q] * a[q] * sc * sc;
      }
    worst[0] = std::max(worst[0], std::sqrt(num0 / std::max(den, 1e-300)));
    worst[1] = std::max(worst[1], std::sqrt(num1 / std::max(den, 1e-300)));
  }
  return (int)orders.size();
}

// CPU restatement of the reference MGPCG Poisson solver and its ghost-fluid
// pressure Strategy.  TEST INFRASTRUCTURE ONLY: this file is the oracle that the
// CUDA path is checked against (tests/, __graft_entry__.smoke()) and the timed
// CPU baseline in bench.py.  No product code path may call it.
//
// Parity status: UNPINNED against the reference itself.  The reference is
// Python on the Taichi DSL and Taichi is not installable offline, so its own
// MGPCG cannot be run.  It ships no tests and no golden vectors.  This
// restatement is pinned instead by (1) scipy sparse direct solves of the same
// assembled system, (2) an independent numpy assembly of A and b, (3) the
// symmetry and linearity of the V-cycle preconditioner (tests/test_oracle.py),
// and (4) a second restatement in vectorised float32 numpy, written from the
// reference's statements, whose system and V-cycle equal this file's bit for
// bit and whose CG loop reaches the same solution
// (tests/test_oracle_numpy_restatement.py).
//
// Followed statement by statement:
//   mgpcg.py:46-60   init_gridtype     (coarse label from 2^d children)
//   mgpcg.py:63-77   initialize        (zero every field)
//   mgpcg.py:79-94   reinitialize / full_reinitialize
//   mgpcg.py:96-102  neighbor_sum
//   mgpcg.py:104-109 smooth            (red-black Gauss-Seidel half sweep)
//   mgpcg.py:111-118 restrict          (unweighted 2^d sum of r - A z)
//   mgpcg.py:120-123 prolongate        (piecewise-constant, unmasked)
//   mgpcg.py:125-148 v_cycle
//   mgpcg.py:150-209 solve             (PCG; squared-norm tolerance)
//   mgpcg.py:211-238 reduce / compute_Ap / update_xr / update_p
//   pressure_project.py:15-39 build_b_kernel (two passes, GFM p0 term)
//   pressure_project.py:45-64 build_A_kernel (GFM 1/theta at level 0 only)
//   utils.py:4-6     FLUID=0, AIR=1, SOLID=2
//
// Rules for what the reference leaves undefined (documented deviations):
//   H1  a neighbour index outside the level grid reads as label SOLID and as
//       value 0 (z, x and Ax); the reference reads out of bounds there.
//   H2  the reference's f32 atomic reductions have no defined order; here
//       `acc_mode` 0 sums sequentially in `Real`, `acc_mode` 1 sums in double.
//       restrict gathers the 2^d children in lexicographic offset order.
//   H3  division by a zero Adiag is not guarded (as in the reference).
//   Level sizes must divide evenly (res % 2^(L-1) == 0); the reference writes
//   out of bounds otherwise.
//
// Build: g++ -O3 -march=native -fopenmp -shared -fPIC (see oracle/build_oracle.py).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum : int8_t { FLUID = 0, AIR = 1, SOLID = 2 };

struct Grid {
  int dim;
  int n[3];          // n[2] == 1 in 2D
  int64_t stride[3]; // row-major, last axis fastest
  int64_t count;
  void init(int d, const int* shape) {
    dim = d;
    n[0] = shape[0];
    n[1] = shape[1];
    n[2] = d == 3 ? shape[2] : 1;
    if (d == 3) {
      stride[2] = 1;
      stride[1] = n[2];
      stride[0] = (int64_t)n[1] * n[2];
    } else {
      stride[1] = 1;
      stride[0] = n[1];
      stride[2] = 0;
    }
    count = (int64_t)n[0] * n[1] * n[2];
  }
  inline void coords(int64_t idx, int c[3]) const {
    if (dim == 3) {
      c[2] = (int)(idx % n[2]);
      int64_t t = idx / n[2];
      c[1] = (int)(t % n[1]);
      c[0] = (int)(t / n[1]);
    } else {
      c[1] = (int)(idx % n[1]);
      c[0] = (int)(idx / n[1]);
      c[2] = 0;
    }
  }
  inline bool in_range(int axis, int v) const { return v >= 0 && v < n[axis]; }
};

template <typename Real>
struct Solver {
  int dim, L, pre_post, bottom;
  std::vector<Grid> g;
  std::vector<std::vector<int8_t>> type;
  std::vector<std::vector<Real>> r, z, Adiag, Ax;  // Ax: dim arrays back to back
  std::vector<Real> b, x, p, Ap;
  Real alpha = 0, beta = 0;  // persistent scalar fields (mgpcg.py:43-44)

  Solver(int d, const int* res, int levels, int pp, int bot)
      : dim(d), L(levels), pre_post(pp), bottom(bot) {
    g.resize(L);
    for (int l = 0; l < L; ++l) {
      int shape[3];
      for (int k = 0; k < d; ++k) shape[k] = res[k] >> l;
      g[l].init(d, shape);
    }
    type.resize(L);
    r.resize(L);
    z.resize(L);
    Adiag.resize(L);
    Ax.resize(L);
    for (int l = 0; l < L; ++l) {
      int64_t c = g[l].count;
      type[l].assign(c, 0);
      r[l].assign(c, 0);
      z[l].assign(c, 0);
      Adiag[l].assign(c, 0);
      Ax[l].assign(c * d, 0);
    }
    int64_t c0 = g[0].count;
    b.assign(c0, 0);
    x.assign(c0, 0);
    p.assign(c0, 0);
    Ap.assign(c0, 0);
  }

  // mgpcg.py:63-77
  void initialize() {
    for (int l = 0; l < L; ++l) {
      std::fill(r[l].begin(), r[l].end(), Real(0));
      std::fill(z[l].begin(), z[l].end(), Real(0));
      std::fill(type[l].begin(), type[l].end(), int8_t(0));
      std::fill(Adiag[l].begin(), Adiag[l].end(), Real(0));
      std::fill(Ax[l].begin(), Ax[l].end(), Real(0));
    }
    std::fill(b.begin(), b.end(), Real(0));
    std::fill(x.begin(), x.end(), Real(0));
    std::fill(p.begin(), p.end(), Real(0));
    std::fill(Ap.begin(), Ap.end(), Real(0));
  }

  // label of the neighbour (H1: out of range reads SOLID)
  inline int8_t nb_type(int l, int64_t idx, const int c[3], int axis, int s) const {
    int v = c[axis] + s;
    if (!g[l].in_range(axis, v)) return SOLID;
    return type[l][idx + s * g[l].stride[axis]];
  }

  // mgpcg.py:46-60 (grid l-1 -> grid l)
  void init_gridtype(int l) {
    const Grid& gf = g[l - 1];
    const Grid& gc = g[l];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gc.count; ++i) {
      int c[3];
      gc.coords(i, c);
      int tot_fluid = 0, tot_air = 0;
      int o2max = dim == 3 ? 2 : 1;
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < o2max; ++o2) {
            int64_t f = (int64_t)(2 * c[0] + o0) * gf.stride[0] +
                        (int64_t)(2 * c[1] + o1) * gf.stride[1] +
                        (dim == 3 ? (int64_t)(2 * c[2] + o2) : 0);
            int attr = type[l - 1][f];
            if (attr == AIR) tot_air++;
            else if (attr == FLUID) tot_fluid++;
          }
      type[l][i] = tot_air > 0 ? AIR : (tot_fluid > 0 ? FLUID : SOLID);
    }
  }

  // mgpcg.py:96-102 with rule H1
  inline Real neighbor_sum(int l, const Real* v, int64_t idx, const int c[3]) const {
    Real ret = Real(0);
    const Grid& gg = g[l];
    const Real* ax = Ax[l].data();
    for (int i = 0; i < dim; ++i) {
      Real lo = Real(0), hi = Real(0);
      if (gg.in_range(i, c[i] - 1)) {
        int64_t j = idx - gg.stride[i];
        lo = ax[i * gg.count + j] * v[j];
      }
      if (gg.in_range(i, c[i] + 1)) {
        int64_t j = idx + gg.stride[i];
        hi = ax[i * gg.count + idx] * v[j];
      }
      ret += lo + hi;
    }
    return ret;
  }

  // mgpcg.py:104-109
  void smooth(int l, int phase) {
    const Grid& gg = g[l];
    Real* zz = z[l].data();
    const Real* rr = r[l].data();
    const Real* ad = Adiag[l].data();
    const int8_t* tt = type[l].data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gg.count; ++i) {
      int c[3];
      gg.coords(i, c);
      if (((c[0] + c[1] + c[2]) & 1) == phase && tt[i] == FLUID)
        zz[i] = (rr[i] - neighbor_sum(l, zz, i, c)) / ad[i];
    }
  }

  // mgpcg.py:111-118, as a gather over the 2^d children (rule H2)
  void restrict_(int l) {
    const Grid& gf = g[l];
    const Grid& gc = g[l + 1];
    const Real* zz = z[l].data();
    const Real* rr = r[l].data();
    const Real* ad = Adiag[l].data();
    const int8_t* tt = type[l].data();
    Real* rc = r[l + 1].data();
#pragma omp parallel for schedule(static)
    for (int64_t ic = 0; ic < gc.count; ++ic) {
      int cc[3];
      gc.coords(ic, cc);
      Real acc = rc[ic];
      int o2max = dim == 3 ? 2 : 1;
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < o2max; ++o2) {
            int c[3] = {2 * cc[0] + o0, 2 * cc[1] + o1, dim == 3 ? 2 * cc[2] + o2 : 0};
            int64_t i = (int64_t)c[0] * gf.stride[0] + (int64_t)c[1] * gf.stride[1] +
                        (dim == 3 ? c[2] : 0);
            if (tt[i] == FLUID) {
              Real Az = ad[i] * zz[i];
              Az += neighbor_sum(l, zz, i, c);
              Real res = rr[i] - Az;
              acc += res;
            }
          }
      rc[ic] = acc;
    }
  }

  // mgpcg.py:120-123
  void prolongate(int l) {
    const Grid& gf = g[l];
    const Grid& gc = g[l + 1];
    Real* zz = z[l].data();
    const Real* zc = z[l + 1].data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gf.count; ++i) {
      int c[3];
      gf.coords(i, c);
      int64_t ic = (int64_t)(c[0] / 2) * gc.stride[0] + (int64_t)(c[1] / 2) * gc.stride[1] +
                   (dim == 3 ? c[2] / 2 : 0);
      zz[i] += zc[ic];
    }
  }

  // mgpcg.py:125-148
  void v_cycle() {
    std::fill(z[0].begin(), z[0].end(), Real(0));
    for (int l = 0; l < L - 1; ++l) {
      for (int i = 0; i < pre_post; ++i) {
        smooth(l, 0);
        smooth(l, 1);
      }
      std::fill(r[l + 1].begin(), r[l + 1].end(), Real(0));
      std::fill(z[l + 1].begin(), z[l + 1].end(), Real(0));
      restrict_(l);
    }
    for (int i = 0; i < bottom / 2; ++i) {
      smooth(L - 1, 0);
      smooth(L - 1, 1);
    }
    for (int i = 0; i < bottom / 2; ++i) {
      smooth(L - 1, 1);
      smooth(L - 1, 0);
    }
    for (int l = L - 2; l >= 0; --l) {
      prolongate(l);
      for (int i = 0; i < pre_post; ++i) {
        smooth(l, 1);
        smooth(l, 0);
      }
    }
  }

  // mgpcg.py:211-216.  acc_mode 0: sequential sum in Real, result rounded to
  // Real (sum[None] is a `real` field); acc_mode 1: double sum, kept in double.
  double reduce(const Real* a, const Real* c, int acc_mode) const {
    const Grid& gg = g[0];
    const int8_t* tt = type[0].data();
    if (acc_mode == 0) {
      Real s = Real(0);
      for (int64_t i = 0; i < gg.count; ++i)
        if (tt[i] == FLUID) s += a[i] * c[i];
      return (double)s;
    }
    // fixed blocks of 4096 cells summed in index order: the same result for
    // any number of threads
    const int64_t B = 4096, nb = (gg.count + B - 1) / B;
    std::vector<double> part(nb, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nb; ++k) {
      double s = 0.0;
      const int64_t e = std::min(gg.count, (k + 1) * B);
      for (int64_t i = k * B; i < e; ++i)
        if (tt[i] == FLUID) s += (double)a[i] * (double)c[i];
      part[k] = s;
    }
    double s = 0.0;
    for (int64_t k = 0; k < nb; ++k) s += part[k];
    return s;
  }

  // mgpcg.py:218-224
  void compute_Ap() {
    const Grid& gg = g[0];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gg.count; ++i) {
      if (type[0][i] == FLUID) {
        int c[3];
        gg.coords(i, c);
        Real v = Adiag[0][i] * p[i];
        v += neighbor_sum(0, p.data(), i, c);
        Ap[i] = v;
      }
    }
  }

  // mgpcg.py:226-232
  void update_xr() {
    const int64_t n = g[0].count;
    const Real a = alpha;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      if (type[0][i] == FLUID) {
        x[i] += a * p[i];
        r[0][i] -= a * Ap[i];
      }
    }
  }

  // mgpcg.py:234-238
  void update_p() {
    const int64_t n = g[0].count;
    const Real bb = beta;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      if (type[0][i] == FLUID) p[i] = z[0][i] + bb * p[i];
  }

  // mgpcg.py:150-209.  Returns the reference's `iter` counter at exit.
  int solve(int max_iters, double rel_tol, double abs_tol, double eps, int acc_mode,
            double* out_rTr0, double* out_rTr, int* out_vcycles) {
    r[0] = b;
    double initial_rTr = reduce(r[0].data(), r[0].data(), acc_mode);
    double tol = std::max(abs_tol, initial_rTr * rel_tol);
    int vcycles = 0;
    v_cycle();
    ++vcycles;
    update_p();
    double old_zTr = reduce(z[0].data(), r[0].data(), acc_mode);
    double rTr = initial_rTr;
    int iter = 0;
    while (max_iters == -1 || iter < max_iters) {
      compute_Ap();
      double pAp = reduce(p.data(), Ap.data(), acc_mode);
      alpha = (Real)(old_zTr / (pAp + eps));
      update_xr();
      rTr = reduce(r[0].data(), r[0].data(), acc_mode);
      if (rTr < tol) break;
      v_cycle();
      ++vcycles;
      double new_zTr = reduce(z[0].data(), r[0].data(), acc_mode);
      beta = (Real)(new_zTr / (old_zTr + eps));
      update_p();
      old_zTr = new_zTr;
      ++iter;
    }
    if (out_rTr0) *out_rTr0 = initial_rTr;
    if (out_rTr) *out_rTr = rTr;
    if (out_vcycles) *out_vcycles = vcycles;
    return iter;
  }

  // pressure_project.py:15-39.  Scalars are kernel constants in the
  // reference and so take the field precision.
  void build_pressure_b(const Real* const* vel, const Real* phi, Real p0, Real scale_A,
                        Real scale_b, int ghost, Real clamp) {
    const Grid& gg = g[0];
    const int8_t* tt = type[0].data();
    // velocity[k] has shape res + e_k
    int64_t vstride[3][3];
    for (int k = 0; k < dim; ++k) {
      int sh[3] = {gg.n[0], gg.n[1], gg.n[2]};
      sh[k] += 1;
      if (dim == 3) {
        vstride[k][2] = 1;
        vstride[k][1] = sh[2];
        vstride[k][0] = (int64_t)sh[1] * sh[2];
      } else {
        vstride[k][1] = 1;
        vstride[k][0] = sh[1];
        vstride[k][2] = 0;
      }
    }
    auto vel_at = [&](int k, const int c[3]) -> Real {
      int64_t o = (int64_t)c[0] * vstride[k][0] + (int64_t)c[1] * vstride[k][1] +
                  (dim == 3 ? (int64_t)c[2] : 0);
      return vel[k][o];
    };
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gg.count; ++i) {
      if (tt[i] != FLUID) continue;
      int c[3];
      gg.coords(i, c);
      Real bi = b[i];
      for (int k = 0; k < dim; ++k) {
        int cp[3] = {c[0], c[1], c[2]};
        cp[k] += 1;
        bi += (vel_at(k, c) - vel_at(k, cp));
      }
      bi *= scale_b;
      b[i] = bi;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gg.count; ++i) {
      if (tt[i] != FLUID) continue;
      int c[3];
      gg.coords(i, c);
      Real bi = b[i];
      for (int k = 0; k < dim; ++k) {
        for (int s = -1; s <= 1; s += 2) {
          int8_t nt = nb_type(0, i, c, k, s);
          if (nt == SOLID) {
            if (s < 0) {
              bi -= scale_b * (vel_at(k, c) - Real(0));
            } else {
              int cp[3] = {c[0], c[1], c[2]};
              cp[k] += 1;
              bi += scale_b * (vel_at(k, cp) - Real(0));
            }
          } else if (nt == AIR) {
            if (ghost) {
              Real phin = phi[i + s * gg.stride[k]];
              Real cc = (phi[i] - phin) / phi[i];
              bi += scale_A * std::min(cc, clamp) * p0;
            } else {
              bi += scale_A * p0;
            }
          }
        }
      }
      b[i] = bi;
    }
  }

  // pressure_project.py:45-64
  void build_pressure_A(int l, const Real* phi, Real scale_A, int ghost, Real clamp) {
    const Grid& gg = g[l];
    const int8_t* tt = type[l].data();
    Real* ad = Adiag[l].data();
    Real* ax = Ax[l].data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < gg.count; ++i) {
      if (tt[i] != FLUID) continue;
      int c[3];
      gg.coords(i, c);
      Real d = ad[i];
      for (int k = 0; k < dim; ++k) {
        for (int s = -1; s <= 1; s += 2) {
          int8_t nt = nb_type(l, i, c, k, s);
          if (nt == FLUID) {
            d += scale_A;
            if (s > 0) ax[k * gg.count + i] = -scale_A;
          } else if (nt == AIR) {
            if (ghost && l == 0) {
              Real phin = phi[i + s * gg.stride[k]];
              Real cc = (phi[i] - phin) / phi[i];
              d += scale_A * std::min(cc, clamp);
            } else {
              d += scale_A;
            }
          }
        }
      }
      ad[i] = d;
    }
  }

  // ---- magnetic potential solve of the 3D substep benchmark --------------
  // Not a reference Strategy: the benchmark's variant of
  // potential_function.py:19-55 (see the CUDA kernels in mg_strategies.cuh).
  static Real mu_face(Real ca, Real cb) {
    Real ma = Real(1) + ca, mb = Real(1) + cb;
    return (Real(2) * (ma * mb)) / (ma + mb);
  }
  bool is_pin(const int c[3], const int pin[3]) const {
    return c[0] == pin[0] && c[1] == pin[1] && (dim == 2 || c[2] == pin[2]);
  }
  void build_psi_b(const Real* chi, const Real H[3], Real dx, const int pin[3]) {
    const Grid& gg = g[0];
    for (int64_t i = 0; i < gg.count; ++i) {
      int c[3];
      gg.coords(i, c);
      if (is_pin(c, pin)) {
        b[i] = Real(0);
        continue;
      }
      Real acc = Real(0);
      for (int k = 0; k < dim; ++k) {
        const int64_t s = gg.stride[k];
        if (c[k] + 1 < gg.n[k]) acc = acc + H[k] * mu_face(chi[i], chi[i + s]);
        if (c[k] > 0) acc = acc - H[k] * mu_face(chi[i - s], chi[i]);
      }
      b[i] = -(acc / dx);
    }
  }
  void build_psi_A0(const Real* chi, Real dx, const int pin[3]) { build_psi_A(0, chi, dx, pin); }
  // level l of the operator from that level's chi and spacing (level 0: the
  // fine chi and dx; rediscretised coarse levels: the children's mean of chi,
  // dx * 2^l, the pin's coarse cell)
  void build_psi_A(int l, const Real* chi, Real dx, const int pin[3]) {
    const Grid& gg = g[l];
    const Real dx2 = dx * dx;
    Real* ad = Adiag[l].data();
    Real* ax = Ax[l].data();
    for (int64_t i = 0; i < gg.count; ++i) {
      int c[3];
      gg.coords(i, c);
      if (is_pin(c, pin)) {
        ad[i] = Real(1) / dx2;
        for (int k = 0; k < dim; ++k) ax[k * gg.count + i] = Real(0);
        continue;
      }
      Real d = Real(0);
      for (int k = 0; k < dim; ++k) {
        const int64_t s = gg.stride[k];
        Real up = Real(0);
        if (c[k] > 0) d = d + mu_face(chi[i - s], chi[i]) / dx2;
        if (c[k] + 1 < gg.n[k]) {
          const Real cf = mu_face(chi[i], chi[i + s]) / dx2;
          d = d + cf;
          int cn[3] = {c[0], c[1], c[2]};
          cn[k] += 1;
          up = is_pin(cn, pin) ? Real(0) : -cf;
        }
        ax[k * gg.count + i] = up;
      }
      ad[i] = d;
    }
  }
  // A_c = scale * P^T A P for piecewise-constant P and child-sum restriction
  void galerkin(int l, Real scale) {
    const Grid& gf = g[l - 1];
    const Grid& gc = g[l];
    for (int64_t ic = 0; ic < gc.count; ++ic) {
      int cc[3];
      gc.coords(ic, cc);
      Real d = Real(0), axc[3] = {Real(0), Real(0), Real(0)};
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < (dim == 3 ? 2 : 1); ++o2) {
            const int o[3] = {o0, o1, o2};
            const int64_t i = (int64_t)(2 * cc[0] + o0) * gf.stride[0] + (int64_t)(2 * cc[1] + o1) * gf.stride[1] +
                              (dim == 3 ? 2 * cc[2] + o2 : 0);
            d = d + Adiag[l - 1][i];
            for (int k = 0; k < dim; ++k) {
              const Real a = Ax[l - 1][k * gf.count + i];
              if (o[k] == 0) d = d + Real(2) * a;
              else axc[k] = axc[k] + a;
            }
          }
      Adiag[l][ic] = scale * d;
      for (int k = 0; k < dim; ++k) Ax[l][k * gc.count + ic] = (cc[k] + 1 < gc.n[k]) ? scale * axc[k] : Real(0);
    }
  }
  // chi of level l: the mean of the 2^dim children of level l-1, summed in
  // lexicographic order from 0 and multiplied by 2^-dim (exact)
  void mean_children(int l, const Real* fine, Real* coarse) const {
    const Grid& gf = g[l - 1];
    const Grid& gc = g[l];
    const Real w = Real(1) / Real(dim == 3 ? 8 : 4);
    for (int64_t ic = 0; ic < gc.count; ++ic) {
      int cc[3];
      gc.coords(ic, cc);
      Real acc = Real(0);
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < (dim == 3 ? 2 : 1); ++o2)
            acc = acc + fine[(int64_t)(2 * cc[0] + o0) * gf.stride[0] + (int64_t)(2 * cc[1] + o1) * gf.stride[1] +
                             (dim == 3 ? 2 * cc[2] + o2 : 0)];
      coarse[ic] = acc * w;
    }
  }
  // full_reinitialize(strategy) (mgpcg.py:89-94) with the potential Strategy;
  // coarse_scale > 0: A_l = coarse_scale * P^T A_(l-1) P; coarse_scale == 0:
  // each coarse level rediscretised as the reference's potential Strategy
  // does (potential_function.py:39-55: chi re-sampled per level, dx * 2^l)
  void full_reinitialize_psi(const Real* chi, const Real H[3], Real dx, const int pin[3], Real coarse_scale) {
    initialize();
    build_psi_b(chi, H, dx, pin);
    for (auto& t : type) std::fill(t.begin(), t.end(), (int8_t)FLUID);
    build_psi_A0(chi, dx, pin);
    if (coarse_scale > Real(0)) {
      for (int l = 1; l < L; ++l) galerkin(l, coarse_scale);
      return;
    }
    std::vector<Real> prev(chi, chi + g[0].count), cur;
    for (int l = 1; l < L; ++l) {
      cur.assign(g[l].count, Real(0));
      mean_children(l, prev.data(), cur.data());
      const int pl[3] = {pin[0] >> l, pin[1] >> l, pin[2] >> l};
      build_psi_A(l, cur.data(), dx * Real(1 << l), pl);
      prev.swap(cur);
    }
  }

  // mgpcg.py:79-87 with the pressure Strategy
  void reinitialize_pressure(const int32_t* cell_type, const Real* const* vel, const Real* phi,
                             Real p0, Real scale_A, Real scale_b, int ghost, Real clamp) {
    initialize();
    for (int64_t i = 0; i < g[0].count; ++i) type[0][i] = (int8_t)cell_type[i];
    build_pressure_b(vel, phi, p0, scale_A, scale_b, ghost, clamp);
    build_pressure_A(0, phi, scale_A, ghost, clamp);
    for (int l = 1; l < L; ++l) {
      init_gridtype(l);
      build_pressure_A(l, phi, scale_A, ghost, clamp);
    }
  }
};

struct Handle {
  int real_bytes;
  void* s;
};

template <typename Real>
Solver<Real>* S(Handle* h) {
  return static_cast<Solver<Real>*>(h->s);
}

enum Field { F_B = 0, F_X = 1, F_P = 2, F_AP = 3, F_R = 4, F_Z = 5, F_ADIAG = 6, F_AX = 7, F_TYPE = 8 };

template <typename Real>
void* field_ptr(Solver<Real>* s, int f, int l, int64_t* count, int* elem) {
  *elem = sizeof(Real);
  *count = s->g[l].count;
  switch (f) {
    case F_B: return s->b.data();
    case F_X: return s->x.data();
    case F_P: return s->p.data();
    case F_AP: return s->Ap.data();
    case F_R: return s->r[l].data();
    case F_Z: return s->z[l].data();
    case F_ADIAG: return s->Adiag[l].data();
    case F_AX: *count = s->g[l].count * s->dim; return s->Ax[l].data();
    case F_TYPE: *elem = 1; return s->type[l].data();
  }
  return nullptr;
}

}  // namespace

#define DISPATCH(h, CALL)                           \
  do {                                              \
    if ((h)->real_bytes == 4) {                     \
      auto* s = S<float>(h);                        \
      CALL;                                         \
    } else {                                        \
      auto* s = S<double>(h);                       \
      CALL;                                         \
    }                                               \
  } while (0)

extern "C" {

// MGPCGPoissonSolver.__init__ (mgpcg.py:6-44); real_bytes 4 = f32, 8 = f64.
void* orc_create(int dim, const int* res, int levels, int pre_post, int bottom, int real_bytes) {
  if (dim != 2 && dim != 3) return nullptr;
  if (real_bytes != 4 && real_bytes != 8) return nullptr;
  for (int k = 0; k < dim; ++k)
    if (res[k] <= 0 || res[k] % (1 << (levels - 1)) != 0) return nullptr;
  Handle* h = new Handle;
  h->real_bytes = real_bytes;
  if (real_bytes == 4) h->s = new Solver<float>(dim, res, levels, pre_post, bottom);
  else h->s = new Solver<double>(dim, res, levels, pre_post, bottom);
  return h;
}

void orc_destroy(void* hh) {
  Handle* h = (Handle*)hh;
  if (!h) return;
  if (h->real_bytes == 4) delete S<float>(h);
  else delete S<double>(h);
  delete h;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Copies between a solver field and a caller buffer of the solver's precision
// (labels are int8).  dir 0: field -> out, dir 1: in -> field.
int orc_field(void* hh, int f, int level, void* buf, int dir) {
  Handle* h = (Handle*)hh;
  int64_t count = 0;
  int elem = 0;
  void* p = nullptr;
  DISPATCH(h, p = field_ptr(s, f, level, &count, &elem));
  if (!p) return -1;
  if (dir == 0) std::memcpy(buf, p, count * elem);
  else std::memcpy(p, buf, count * elem);
  return 0;
}

void orc_initialize(void* hh) { Handle* h = (Handle*)hh; DISPATCH(h, s->initialize()); }
void orc_init_gridtype(void* hh, int l) { Handle* h = (Handle*)hh; DISPATCH(h, s->init_gridtype(l)); }
void orc_smooth(void* hh, int l, int phase) { Handle* h = (Handle*)hh; DISPATCH(h, s->smooth(l, phase)); }
void orc_restrict(void* hh, int l) { Handle* h = (Handle*)hh; DISPATCH(h, s->restrict_(l)); }
void orc_prolongate(void* hh, int l) { Handle* h = (Handle*)hh; DISPATCH(h, s->prolongate(l)); }
void orc_v_cycle(void* hh) { Handle* h = (Handle*)hh; DISPATCH(h, s->v_cycle()); }
void orc_compute_Ap(void* hh) { Handle* h = (Handle*)hh; DISPATCH(h, s->compute_Ap()); }

// Fills every level's labels with FLUID (mgpcg.py:93, full_reinitialize).
void orc_fill_fluid(void* hh) {
  Handle* h = (Handle*)hh;
  DISPATCH(h, for (auto& t : s->type) std::fill(t.begin(), t.end(), (int8_t)FLUID));
}

// reinitialize(cell_type, PressureProjectStrategy); vel/phi in the solver's
// precision, cell_type int32 (the simulator's field type).
void orc_reinitialize_pressure(void* hh, const int32_t* cell_type, const void* const* vel,
                               const void* phi, double p0, double scale_A, double scale_b,
                               int ghost, double clamp) {
  Handle* h = (Handle*)hh;
  if (h->real_bytes == 4) {
    auto* s = S<float>(h);
    s->reinitialize_pressure(cell_type, (const float* const*)vel, (const float*)phi, (float)p0,
                             (float)scale_A, (float)scale_b, ghost, (float)clamp);
  } else {
    auto* s = S<double>(h);
    s->reinitialize_pressure(cell_type, (const double* const*)vel, (const double*)phi, p0,
                             scale_A, scale_b, ghost, clamp);
  }
}

// full_reinitialize with the magnetic potential Strategy; chi in the solver's precision.
void orc_full_reinitialize_psi(void* hh, const void* chi, double H0, double H1, double H2, double dx, int p0,
                               int p1, int p2, double coarse_scale) {
  Handle* h = (Handle*)hh;
  const int pin[3] = {p0, p1, p2};
  if (h->real_bytes == 4) {
    const float H[3] = {(float)H0, (float)H1, (float)H2};
    S<float>(h)->full_reinitialize_psi((const float*)chi, H, (float)dx, pin, (float)coarse_scale);
  } else {
    const double H[3] = {H0, H1, H2};
    S<double>(h)->full_reinitialize_psi((const double*)chi, H, dx, pin, coarse_scale);
  }
}

double orc_reduce(void* hh, int fa, int fb, int acc_mode) {
  Handle* h = (Handle*)hh;
  double out = 0;
  DISPATCH(h, {
    int64_t c;
    int e;
    auto* a = (decltype(s->b.data()))field_ptr(s, fa, 0, &c, &e);
    auto* b = (decltype(s->b.data()))field_ptr(s, fb, 0, &c, &e);
    out = s->reduce(a, b, acc_mode);
  });
  return out;
}

// solve(max_iters, rel_tol, abs_tol, eps) (mgpcg.py:150-209).
int orc_solve(void* hh, int max_iters, double rel_tol, double abs_tol, double eps, int acc_mode,
              double* out_rTr0, double* out_rTr, int* out_vcycles) {
  Handle* h = (Handle*)hh;
  int it = 0;
  DISPATCH(h, it = s->solve(max_iters, rel_tol, abs_tol, eps, acc_mode, out_rTr0, out_rTr,
                            out_vcycles));
  return it;
}

}  // extern "C"

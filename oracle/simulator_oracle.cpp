// CPU restatement of the reference's other Poisson Strategies and of the
// pressure-gradient step after the solve.  TEST INFRASTRUCTURE ONLY: the
// oracle the CUDA kernels of these rows are checked against (tests/).  No
// product code path may call it.
//
// Parity status: UNPINNED against the reference itself (Taichi is not
// installable offline, and the reference ships no tests for these files).
// Pinned instead by hand-computed cases and structural properties in
// tests/test_oracle_strategies.py (symmetry of the assembled operators,
// sampling identities, volume of known shapes, momentum identities of the
// pressure update).
//
// Followed statement by statement, all arithmetic in f32 with one IEEE
// rounding per written operation (compiled with -ffp-contract=off):
//   utils.py:12-33                    sample (bi/trilinear, clamped)
//   level_set.py:24-37                theta / delta (smoothed Heaviside, Dirac)
//   fluid_simulator.py:123-136        is_valid / is_fluid / is_solid / is_air
//   fluid_simulator.py:193-214        apply_pressure
//   ferrofluid_simulator.py:64-69     H_interp
//   ferrofluid_simulator.py:115-137   apply_magnetic_force
//   magnetic_force.py:17-38           MagneticForceStrategy.build_b_kernel
//   potential_function.py:15-55       PotentialFunctionStrategy
//   volume_control.py:22-51           calc_volume, add_c and the PI controller
//   surface_tension.py:23-95, 108-129 SurfaceTensionStrategy, calc_n, calc_kappa
//   level_set.py:114-163, 266-392     markers: distance, propagation, target_minus,
//                                     smoothing (FastSweepingLevelSet.build_from_markers)
// Constants the reference computes in Python double before they meet f32
// values are passed in already folded (the caller folds them in double).
// Rule H1 of the solver oracle holds here too: a label outside the grid is
// SOLID.  The volume is summed over cells in double (the reference sums f32
// atomically in an undefined order).

#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

namespace {

enum : int { FLUID = 0, AIR = 1, SOLID = 2 };

struct G {
  int dim;
  int n[3];  // n[2] == 1 in 2D
  int64_t cells() const { return (int64_t)n[0] * n[1] * n[2]; }
  int64_t at(int i, int j, int k) const { return ((int64_t)i * n[1] + j) * n[2] + k; }
};

G make(int dim, const int* res) {
  G g;
  g.dim = dim;
  g.n[0] = res[0];
  g.n[1] = res[1];
  g.n[2] = dim == 3 ? res[2] : 1;
  return g;
}

// Shape of the MAC face field of axis k: res + e_k.
G faces(const G& c, int k) {
  G g = c;
  g.n[k] += 1;
  return g;
}

int clampi(int v, int a, int b) { return v < a ? a : (v > b ? b : v); }
float clampf(float v, float a, float b) { return std::fmax(a, std::fmin(b, v)); }

// utils.sample: int() truncates toward zero; indices and weights clamped.
float sample(const float* d, const G& g, const float* pos) {
  int i = clampi((int)pos[0], 0, g.n[0] - 1), j = clampi((int)pos[1], 0, g.n[1] - 1);
  int ip = clampi(i + 1, 0, g.n[0] - 1), jp = clampi(j + 1, 0, g.n[1] - 1);
  float s = clampf(pos[0] - (float)i, 0.0f, 1.0f), t = clampf(pos[1] - (float)j, 0.0f, 1.0f);
  if (g.dim == 2) {
    float lo = d[g.at(i, j, 0)] * (1.0f - s) + d[g.at(ip, j, 0)] * s;
    float hi = d[g.at(i, jp, 0)] * (1.0f - s) + d[g.at(ip, jp, 0)] * s;
    return lo * (1.0f - t) + hi * t;
  }
  int k = clampi((int)pos[2], 0, g.n[2] - 1), kp = clampi(k + 1, 0, g.n[2] - 1);
  float u = clampf(pos[2] - (float)k, 0.0f, 1.0f);
  float a = d[g.at(i, j, k)] * (1.0f - s) + d[g.at(ip, j, k)] * s;
  float b = d[g.at(i, jp, k)] * (1.0f - s) + d[g.at(ip, jp, k)] * s;
  float c = d[g.at(i, j, kp)] * (1.0f - s) + d[g.at(ip, j, kp)] * s;
  float e = d[g.at(i, jp, kp)] * (1.0f - s) + d[g.at(ip, jp, kp)] * s;
  return (a * (1.0f - t) + b * t) * (1.0f - u) + (c * (1.0f - t) + e * t) * u;
}

struct Eps {
  float eps, two_eps, pi, inv_2pi;
};

Eps eps_consts(double eps) {
  const double pi = 3.14159265358979323846;
  return Eps{(float)eps, (float)(2.0 * eps), (float)pi, (float)(1.0 / (2.0 * pi))};
}

float theta(float phi, const Eps& e) {
  if (phi <= -e.eps) return 0.0f;
  if (phi >= e.eps) return 1.0f;
  return 0.5f + phi / e.two_eps + e.inv_2pi * std::sin(e.pi * phi / e.eps);
}

float delta(float phi, const Eps& e) {
  if (phi <= -e.eps || phi >= e.eps) return 0.0f;
  return (1.0f + std::cos(e.pi * phi / e.eps)) / e.two_eps;
}

void coords(const G& g, int64_t idx, int c[3]) {
  c[2] = (int)(idx % g.n[2]);
  int64_t t = idx / g.n[2];
  c[1] = (int)(t % g.n[1]);
  c[0] = (int)(t / g.n[1]);
}

bool valid(const G& g, const int c[3]) {
  for (int a = 0; a < g.dim; ++a)
    if (c[a] < 0 || c[a] >= g.n[a]) return false;
  return true;
}

// |H_interp(c + 0.5)|^2 with H the MAC field (one array per axis).
float h2(const float* const* H, const G& g, const int c[3]) {
  float acc = 0.0f;
  for (int q = 0; q < g.dim; ++q) {
    float pos[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < g.dim; ++a) pos[a] = ((float)c[a] + 0.5f) - (a == q ? 0.0f : 0.5f);
    float h = sample(H[q], faces(g, q), pos);
    acc = acc + h * h;
  }
  return acc;
}

}  // namespace

extern "C" {

// apply_pressure (H == nullptr) or apply_magnetic_force (H given), all axes.
void ors_apply_pressure(int dim, const int* res, float* const* u, const float* p, const int32_t* ct,
                        const float* phi, float scale, float p0, int ghost, float clamp, const float* const* H,
                        float coef) {
  const G g = make(dim, res);
  for (int k = 0; k < dim; ++k) {
    const G f = faces(g, k);
    for (int64_t i = 0; i < g.cells(); ++i) {
      int c[3], c1[3];
      coords(g, i, c);
      for (int a = 0; a < 3; ++a) c1[a] = c[a];
      c1[k] -= 1;
      const bool v1 = valid(g, c1);
      const int64_t i1 = v1 ? g.at(c1[0], c1[1], c1[2]) : -1;
      const bool fluid = ct[i] == FLUID, fluid1 = v1 && ct[i1] == FLUID;
      const bool solid = ct[i] == SOLID, solid1 = !v1 || ct[i1] == SOLID;
      const bool air = ct[i] == AIR, air1 = v1 && ct[i1] == AIR;
      if (!(fluid1 || fluid)) continue;
      float& uf = u[k][f.at(c[0], c[1], c[2])];
      if (solid1 || solid) {
        uf = 0.0f;
      } else if (air) {
        if (H) {
          uf -= scale * ((p0 + coef * h2(H, g, c)) - p[i1]);
        } else if (ghost) {
          float cc = (phi[i1] - phi[i]) / phi[i1];
          uf -= scale * (p0 - p[i1]) * std::fmin(cc, clamp);
        } else {
          uf -= scale * (p0 - p[i1]);
        }
      } else if (air1) {
        if (H) {
          uf -= scale * (p[i] - (p0 + coef * h2(H, g, c1)));
        } else if (ghost) {
          float cc = (phi[i] - phi[i1]) / phi[i];
          uf -= scale * (p[i] - p0) * std::fmin(cc, clamp);
        } else {
          uf -= scale * (p[i] - p0);
        }
      } else {
        uf -= scale * (p[i] - p[i1]);
      }
    }
  }
}

// calc_volume: sum over cells of the corner mean of theta(-phi(corner)).
double ors_volume(int dim, const int* res, const float* phi, double eps) {
  const G g = make(dim, res);
  const Eps e = eps_consts(eps);
  const int corners = 1 << dim;
  double vol = 0.0;
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    float cell = 0.0f;
    for (int o = 0; o < corners; ++o) {  // row-major offsets, last axis fastest
      int off[3] = {0, 0, 0};
      for (int a = 0; a < dim; ++a) off[a] = (o >> (dim - 1 - a)) & 1;
      float pos[3];
      for (int a = 0; a < 3; ++a) pos[a] = (float)(c[a] + off[a]) - 0.5f;
      cell = cell + theta(-sample(phi, g, pos), e);
    }
    vol += (double)(cell / (float)corners);
  }
  return vol;
}

// One volume-control build_b step after the pressure build_b: the controller
// state (FP64) [0] step, [1] vol_0, [2] y, [3] vol, [4] c, [5] k_p, [6] k_i,
// [7] dt, then b += (f32)c on FLUID cells from the second step on.
void ors_volume_control(int dim, const int* res, const float* phi, double eps, const int8_t* type, float* b,
                        double* st) {
  const G g = make(dim, res);
  const double vol = ors_volume(dim, res, phi, eps);
  st[0] += 1.0;
  st[3] = vol;
  if (st[0] == 1.0) {
    st[1] = vol;
    return;
  }
  const double x = (vol - st[1]) / st[1];
  st[2] += x * st[7];
  st[4] = (-st[5] * x - st[6] * st[2]) / (x + 1.0);
  const float c = (float)st[4];
  for (int64_t i = 0; i < g.cells(); ++i)
    if (type[i] == FLUID) b[i] += c;
}

// MagneticForceStrategy.build_b_kernel on level 0 (b zeroed by the caller
// through initialize).  type: the level-0 labels (int8).
void ors_build_magnetic_b(int dim, const int* res, const int8_t* type, const float* const* v,
                          const float* const* H, float p0, float sA, float sB, float coef, float* b) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {  // pass 1
    if (type[i] != FLUID) continue;
    int c[3];
    coords(g, i, c);
    for (int k = 0; k < dim; ++k) {
      const G f = faces(g, k);
      b[i] += v[k][f.at(c[0], c[1], c[2])] - v[k][f.at(c[0] + (k == 0), c[1] + (k == 1), c[2] + (k == 2))];
    }
    b[i] *= sB;
  }
  for (int64_t i = 0; i < g.cells(); ++i) {  // pass 2
    if (type[i] != FLUID) continue;
    int c[3];
    coords(g, i, c);
    for (int k = 0; k < dim; ++k) {
      const G f = faces(g, k);
      for (int s = -1; s <= 1; s += 2) {
        int cn[3] = {c[0], c[1], c[2]};
        cn[k] += s;
        const int t = valid(g, cn) ? type[g.at(cn[0], cn[1], cn[2])] : SOLID;
        if (t == SOLID) {
          if (s < 0) b[i] -= sB * (v[k][f.at(c[0], c[1], c[2])] - 0.0f);
          else b[i] += sB * (v[k][f.at(cn[0], cn[1], cn[2])] - 0.0f);
        } else if (t == AIR) {
          b[i] += sA * (p0 + coef * h2(H, g, cn));
        }
      }
    }
  }
}

// PotentialFunctionStrategy: in_domain tests against the fine res.
static bool in_domain(int dim, const int* res, const int c[3]) {
  for (int a = 0; a < dim; ++a)
    if (!(c[a] >= 0 && c[a] + 1 <= res[a])) return false;
  return true;
}

void ors_build_potential_b(int dim, const int* res, const float* chi, const float* const* Hext, float* b) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    bool origin = true;
    for (int a = 0; a < dim; ++a) origin = origin && c[a] == 0;
    if (origin) {
      b[i] = 0.0f;
      continue;
    }
    if (!in_domain(dim, res, c)) continue;
    for (int k = 0; k < dim; ++k) {
      const G f = faces(g, k);
      int up[3] = {c[0], c[1], c[2]}, dn[3] = {c[0], c[1], c[2]};
      up[k] += 1;
      dn[k] -= 1;
      if (in_domain(dim, res, up)) {
        float pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = (float)up[a] + (a == k ? 0.0f : 0.5f);
        b[i] += sample(chi, g, pos) * Hext[k][f.at(up[0], up[1], up[2])];
      }
      if (in_domain(dim, res, dn)) {
        float pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = (float)c[a] + (a == k ? 0.0f : 0.5f);
        b[i] -= sample(chi, g, pos) * Hext[k][f.at(c[0], c[1], c[2])];
      }
    }
  }
}

// One level (shape res >> level) of the potential operator; Adiag and Ax
// (dim planes) zeroed by the caller.  chi has the fine shape res.
void ors_build_potential_A(int dim, const int* res, int level, const float* chi, double dx, float* Adiag,
                           float* Ax) {
  const G fine = make(dim, res);
  int rl[3] = {res[0] >> level, res[1] >> level, dim == 3 ? res[2] >> level : 1};
  const G g = make(dim, rl);
  const double dxl = dx * (double)(1 << level);
  const float fdx = (float)dxl, inv = (float)(1.0 / dxl), m = (float)(1 << level);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    bool origin = true;
    for (int a = 0; a < dim; ++a) origin = origin && c[a] == 0;
    if (origin) {
      Adiag[i] = inv;
      continue;
    }
    if (!in_domain(dim, res, c)) continue;
    for (int k = 0; k < dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        int cn[3] = {c[0], c[1], c[2]};
        cn[k] += s;
        if (!in_domain(dim, res, cn)) continue;
        float pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = ((float)c[a] + (a == k ? 0.5f * (float)s : 0.0f)) * m;
        const float cf = (1.0f + sample(chi, fine, pos)) / fdx;
        Adiag[i] -= cf;
        if (s > 0) Ax[k * g.cells() + i] = cf;
      }
  }
}

// LevelSet.initialize_with_aabb / initialize_with_sphere (level_set.py:40-64)
// at cell centres (I + 0.5) dx; combine: min with the existing phi.
void ors_level_set_shape(int dim, const int* res, float* phi, float dx, int sphere, const float* a, const float* b,
                         int combine) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    float x[3];
    for (int k = 0; k < dim; ++k) x[k] = ((float)c[k] + 0.5f) * dx;
    float v;
    if (sphere) {
      float s = 0.0f;
      for (int k = 0; k < dim; ++k) {
        const float d = x[k] - a[k];
        s = k == 0 ? d * d : s + d * d;
      }
      v = std::sqrt(s) - b[0];
    } else {
      bool inside = true;
      for (int k = 0; k < dim; ++k) inside = inside && x[k] > a[k] && x[k] < b[k];
      if (inside) {
        v = std::fmax(a[0] - x[0], x[0] - b[0]);
        for (int k = 1; k < dim; ++k) v = std::fmax(v, std::fmax(a[k] - x[k], x[k] - b[k]));
      } else {
        float s = 0.0f;
        for (int k = 0; k < dim; ++k) {
          const float p = x[k] < a[k] ? a[k] : (x[k] > b[k] ? b[k] : x[k]);
          const float d = x[k] - p;
          s = k == 0 ? d * d : s + d * d;
        }
        v = std::sqrt(s);
      }
    }
    phi[i] = combine ? std::fmin(phi[i], v) : v;
  }
}

// FluidSimulator.apply_markers (fluid_simulator.py:151-159).
void ors_apply_markers(int dim, const int* res, int32_t* ct, const float* phi, int strict) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i)
    if (ct[i] != SOLID) ct[i] = AIR;
  for (int64_t i = 0; i < g.cells(); ++i)
    if (ct[i] != SOLID && (strict ? phi[i] < 0.0f : phi[i] <= 0.0f)) ct[i] = FLUID;
}

// FluidSimulator.init_boundary (fluid_simulator.py:337-341).
void ors_init_boundary(int dim, const int* res, int32_t* ct) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    bool edge = false;
    for (int k = 0; k < dim; ++k) edge = edge || c[k] == 0 || c[k] + 1 == g.n[k];
    if (edge) ct[i] = SOLID;
  }
}

// FastSweepingLevelSet.redistance (level_set.py:260-334) with target_surface
// (:66-86) and update_from_neighbor (:88-112).  ts.sign is GLSL's sign
// (-1, 0, +1) as in taichi_glsl (a dependency absent here, version
// unpinned).  The reference runs the lines of a sweep in parallel; this runs
// them one after another in index order, which is one of its schedules.
// The reference bounds the forward axis-0 sweeps by res[1]
// (level_set.py:303, 322); here res[0] (the same on square / cubic grids).
static float gsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// FastSweepingLevelSet.propagate (level_set.py:266-327): repeat rounds of the
// 2 dim sweeps (fastest axis first, forward then backward), each line walked
// in order, update_from_neighbor (level_set.py:88-112) on every cell whose
// valid is -1; t holds phi_temp, phi gives the sign.  Lines one after another
// (the reference runs them in parallel, reading each other's cells).
static void fs_propagate(const G& g, const float* phi, float* t, const int32_t* valid, double dx, int repeat) {
  const int dim = g.dim;
  const int64_t n = g.cells();
  const float fdx = (float)dx, two_dx2 = (float)(2.0 * dx * dx), dx2 = (float)(dx * dx), third = (float)(1.0 / 3.0);
  auto stride = [&](int k) -> int64_t { return k == 0 ? (int64_t)g.n[1] * g.n[2] : (k == 1 ? g.n[2] : 1); };
  auto update = [&](int64_t i, const int c[3]) {
    float nb[3];
    for (int k = 0; k < dim; ++k) {
      const int64_t st = stride(k);
      if (c[k] == 0 || (c[k] < g.n[k] - 1 && std::fabs(t[i + st]) < std::fabs(t[i - st]))) nb[k] = std::fabs(t[i + st]);
      else nb[k] = std::fabs(t[i - st]);
    }
    for (int a = 0; a < dim - 1; ++a)
      for (int b = 0; b < dim - 1 - a; ++b)
        if (nb[b] > nb[b + 1]) std::swap(nb[b], nb[b + 1]);
    float d = nb[0] + fdx;
    if (d > nb[1]) {
      const float e = nb[1] - nb[0];
      d = 0.5f * (nb[0] + nb[1] + std::sqrt(two_dx2 - e * e));
      if (dim == 3 && d > nb[2]) {
        const float s = nb[0] + nb[1] + nb[2];
        const float q = nb[0] * nb[0] + nb[1] * nb[1] + nb[2] * nb[2] - dx2;
        d = third * (s + std::sqrt(std::fmax(0.0f, s * s - 3.0f * q)));
      }
    }
    if (std::fabs(d) < std::fabs(t[i])) t[i] = d * gsign(phi[i]);
  };
  for (int r = 0; r < repeat; ++r)
    for (int axis = dim - 1; axis >= 0; --axis)
      for (int dir = 1; dir >= -1; dir -= 2) {
        int oa[2], no = 0;
        for (int k = 0; k < dim; ++k)
          if (k != axis) oa[no++] = k;
        const int64_t lines = n / g.n[axis];
        const int nfast = no == 2 ? g.n[oa[1]] : 1;
        for (int64_t l = 0; l < lines; ++l) {
          int c[3] = {0, 0, 0};
          if (no == 2) {
            c[oa[0]] = (int)(l / nfast);
            c[oa[1]] = (int)(l % nfast);
          } else {
            c[oa[0]] = (int)l;
          }
          for (int step = 0; step < g.n[axis]; ++step) {
            c[axis] = dir > 0 ? step : g.n[axis] - 1 - step;
            const int64_t i = g.at(c[0], c[1], c[2]);
            if (valid[i] == -1) update(i, c);
          }
        }
      }
}

void ors_redistance(int dim, const int* res, float* phi, double dx, int repeat, float* temp_out, int32_t* valid_out) {
  const G g = make(dim, res);
  const int64_t n = g.cells();
  std::vector<float> t(n);
  std::vector<int32_t> valid(n, -1);
  const float fdx = (float)dx;
  auto stride = [&](int k) -> int64_t { return k == 0 ? (int64_t)g.n[1] * g.n[2] : (k == 1 ? g.n[2] : 1); };
  for (int64_t i = 0; i < n; ++i) {  // target_surface
    int c[3];
    coords(g, i, c);
    const float p = phi[i], sp = gsign(p);
    bool change = false;
    float est = 1e20f;
    for (int k = 0; k < dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v < 0 || v >= g.n[k]) continue;
        const float q = phi[i + s * stride(k)];
        if (sp != gsign(q)) {
          const float theta = p / (p - q);
          const float est0 = sp * theta * fdx;
          est = std::fabs(est0) < std::fabs(est) ? est0 : est;
          change = true;
        }
      }
    t[i] = change ? est : 1e20f;
    if (change) valid[i] = 0;
  }
  fs_propagate(g, phi, t.data(), valid.data(), dx, repeat);
  for (int64_t i = 0; i < n; ++i) {
    phi[i] = t[i];
    if (temp_out) temp_out[i] = t[i];
    if (valid_out) valid_out[i] = valid[i];
  }
}

// The cell of a marker (coordinates / dx truncated toward zero, the
// reference's cast) and its distance to the cell centre (I + 0.5) dx; false
// when the cell is outside the grid or a coordinate is not finite.
static bool marker_cell(const G& g, const float* m, float dx, int c[3], float* d) {
  float s = 0.0f;
  bool in = true;
  c[0] = c[1] = c[2] = 0;
  for (int a = 0; a < g.dim; ++a) {
    const float q = m[a] / dx;
    if (!std::isfinite(q) || std::fabs(q) > 2.0e9f) return false;
    const int I = (int)q;
    c[a] = I;
    in = in && I >= 0 && I < g.n[a];
    const float diff = m[a] - ((float)I + 0.5f) * dx;
    s = a == 0 ? diff * diff : s + diff * diff;
  }
  *d = std::sqrt(s);
  return in;
}

// FastSweepingLevelSet.build_from_markers, first part (level_set.py:381-385):
// phi = 1e20, valid = -1, distance_to_markers (level_set.py:114-122; markers
// in index order, a cell keeps the smallest distance and the first marker
// reaching it - the reference's parallel loop races between markers of one
// cell), then markers_propagate (level_set.py:336-379): repeat rounds of the
// 2 dim sweeps, each line walked in order, a cell taking the distance to the
// marker of its neighbour one step ahead when smaller.  A neighbour without a
// marker (valid -1) is skipped: the reference indexes markers[-1] there.
void ors_markers_distance(int dim, const int* res, const float* markers, int n_markers, float dx, int repeat,
                          float* phi, int32_t* valid) {
  const G g = make(dim, res);
  const int64_t n = g.cells();
  for (int64_t i = 0; i < n; ++i) {
    phi[i] = 1e20f;
    valid[i] = -1;
  }
  for (int p = 0; p < n_markers; ++p) {
    int c[3];
    float d;
    if (!marker_cell(g, markers + (int64_t)p * dim, dx, c, &d)) continue;
    const int64_t i = g.at(c[0], c[1], c[2]);
    if (d < phi[i]) {
      phi[i] = d;
      valid[i] = p;
    }
  }
  for (int r = 0; r < repeat; ++r)
    for (int axis = dim - 1; axis >= 0; --axis)
      for (int dir = 1; dir >= -1; dir -= 2) {
        int oa[2], no = 0;
        for (int k = 0; k < dim; ++k)
          if (k != axis) oa[no++] = k;
        const int64_t lines = n / g.n[axis];
        const int nfast = no == 2 ? g.n[oa[1]] : 1;
        for (int64_t l = 0; l < lines; ++l) {
          int c[3] = {0, 0, 0};
          if (no == 2) {
            c[oa[0]] = (int)(l / nfast);
            c[oa[1]] = (int)(l % nfast);
          } else {
            c[oa[0]] = (int)l;
          }
          for (int step = 0; step < g.n[axis]; ++step) {
            c[axis] = dir > 0 ? step : g.n[axis] - 1 - step;
            int nc[3] = {c[0], c[1], c[2]};
            nc[axis] += dir;
            if (nc[axis] < 0 || nc[axis] >= g.n[axis]) continue;
            const int32_t v = valid[g.at(nc[0], nc[1], nc[2])];
            if (v < 0) continue;
            float s = 0.0f;
            for (int a = 0; a < dim; ++a) {
              const float diff = markers[(int64_t)v * dim + a] - ((float)c[a] + 0.5f) * dx;
              s = a == 0 ? diff * diff : s + diff * diff;
            }
            const float d = std::sqrt(s);
            const int64_t i = g.at(c[0], c[1], c[2]);
            if (d < phi[i]) {
              phi[i] = d;
              valid[i] = v;
            }
          }
        }
      }
}

// LevelSet.target_minus (level_set.py:124-146) after valid.fill(-1): phi -= r
// (r = 0.99 dx folded in double), then cells on the interface side of a sign
// change with phi <= 0 are known (valid 0, phi_temp = phi), other phi <= 0
// cells get phi_temp = -1 (to be swept), phi > 0 cells are known.
void ors_target_minus(int dim, const int* res, float* phi, float r, float* phi_temp, int32_t* valid) {
  const G g = make(dim, res);
  const int64_t n = g.cells();
  auto stride = [&](int k) -> int64_t { return k == 0 ? (int64_t)g.n[1] * g.n[2] : (k == 1 ? g.n[2] : 1); };
  for (int64_t i = 0; i < n; ++i) {
    phi[i] = phi[i] - r;
    valid[i] = -1;
  }
  for (int64_t i = 0; i < n; ++i) {
    int c[3];
    coords(g, i, c);
    bool change = false;
    for (int k = 0; k < dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v >= 0 && v < g.n[k] && gsign(phi[i]) != gsign(phi[i + s * stride(k)])) change = true;
      }
    if (change && phi[i] <= 0.0f) {
      valid[i] = 0;
      phi_temp[i] = phi[i];
    } else if (phi[i] <= 0.0f) {
      phi_temp[i] = -1.0f;
    } else {
      phi_temp[i] = phi[i];
      valid[i] = 0;
    }
  }
}

// FastSweepingLevelSet.propagate alone (the sweeps of redistance).
void ors_fs_propagate(int dim, const int* res, const float* phi, float* phi_temp, const int32_t* valid, double dx,
                      int repeat) {
  fs_propagate(make(dim, res), phi, phi_temp, valid, dx, repeat);
}

// LevelSet.smoothing (level_set.py:148-163): out = min(mean of the in-range
// axis neighbours of in (summed axis by axis, lower then upper), in).
void ors_ls_smooth(int dim, const int* res, float* out, const float* in) {
  const G g = make(dim, res);
  const int64_t n = g.cells();
  auto stride = [&](int k) -> int64_t { return k == 0 ? (int64_t)g.n[1] * g.n[2] : (k == 1 ? g.n[2] : 1); };
  for (int64_t i = 0; i < n; ++i) {
    int c[3];
    coords(g, i, c);
    float avg = 0.0f;
    int tot = 0;
    for (int k = 0; k < dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v >= 0 && v < g.n[k]) {
          avg = avg + in[i + s * stride(k)];
          ++tot;
        }
      }
    avg = avg / (float)tot;
    out[i] = avg < in[i] ? avg : in[i];
  }
}

// FluidSimulator.vel_interp (fluid_simulator.py:138-143).
static void vel_interp(const float* const* u, const G& g, float dx, const float* pos, float* v) {
  for (int q = 0; q < g.dim; ++q) {
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < g.dim; ++a) s[a] = pos[a] / dx - (a == q ? 0.0f : 0.5f);
    v[q] = sample(u[q], faces(g, q), s);
  }
}

// FluidSimulator.advect (fluid_simulator.py:216-221) of one field: field -1
// the cell field (offset 0.5), field k the faces of axis k (0.5 (1 - e_k)).
void ors_advect(int dim, const int* res, const float* const* u, int field, const float* src, float* dst, float dx,
                float dt) {
  const G g = make(dim, res);
  const G f = field < 0 ? g : faces(g, field);
  const float half_dt = 0.5f * dt;
  for (int64_t i = 0; i < f.cells(); ++i) {
    int c[3];
    coords(f, i, c);
    float off[3], pos[3], v[3], mid[3], p0[3], s[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < 3; ++a) off[a] = (a >= dim || (field >= 0 && a == field)) ? 0.0f : 0.5f;
    for (int a = 0; a < dim; ++a) pos[a] = ((float)c[a] + off[a]) * dx;
    vel_interp(u, g, dx, pos, v);
    for (int a = 0; a < dim; ++a) mid[a] = pos[a] - v[a] * half_dt;
    vel_interp(u, g, dx, mid, v);
    for (int a = 0; a < dim; ++a) p0[a] = pos[a] - v[a] * dt;
    for (int a = 0; a < dim; ++a) s[a] = p0[a] / dx - off[a];
    dst[i] = sample(src, f, s);
  }
}

// FluidSimulator.extrap_velocity for axis k (fluid_simulator.py:244-272): the
// valid faces, then `iterations` rounds of diffuse_quantity (a neighbour
// outside the face array is invalid).
void ors_extrapolate(int dim, const int* res, int k, float* u, const int32_t* ct, int iterations, int32_t* valid_out) {
  const G g = make(dim, res);
  const G f = faces(g, k);
  const int64_t n = f.cells();
  std::vector<int32_t> valid(n), vt(n);
  std::vector<float> backup(n);
  for (int64_t i = 0; i < n; ++i) {
    int c[3];
    coords(f, i, c);
    int c1[3] = {c[0], c[1], c[2]};
    c1[k] -= 1;
    const bool fl1 = c1[k] >= 0 && ct[g.at(c1[0], c1[1], c1[2])] == FLUID;
    const bool fl0 = c[k] < g.n[k] && ct[g.at(c[0], c[1], c[2])] == FLUID;
    valid[i] = (fl1 || fl0) ? 1 : 0;
  }
  const int span = dim == 3 ? 27 : 9;
  for (int it = 0; it < iterations; ++it) {
    for (int64_t i = 0; i < n; ++i) {
      backup[i] = u[i];
      vt[i] = valid[i];
    }
    for (int64_t i = 0; i < n; ++i) {
      if (vt[i] != 0) continue;
      int c[3];
      coords(f, i, c);
      float tot = 0.0f;
      int cnt = 0;
      for (int o = 0; o < span; ++o) {
        int m[3] = {c[0], c[1], c[2]};
        if (dim == 3) {
          m[0] += o / 9 - 1;
          m[1] += (o / 3) % 3 - 1;
          m[2] += o % 3 - 1;
        } else {
          m[0] += o / 3 - 1;
          m[1] += o % 3 - 1;
        }
        bool in = true;
        for (int a = 0; a < dim; ++a) in = in && m[a] >= 0 && m[a] < f.n[a];
        if (!in) continue;
        const int64_t j = f.at(m[0], m[1], m[2]);
        if (vt[j] == 1) {
          tot += backup[j];
          ++cnt;
        }
      }
      if (cnt > 0) {
        u[i] = tot / (float)cnt;
        valid[i] = 1;
      }
    }
  }
  if (valid_out)
    for (int64_t i = 0; i < n; ++i) valid_out[i] = valid[i];
}

// FluidSimulator.enforce_boundary (fluid_simulator.py:168-174).
void ors_enforce_boundary(int dim, const int* res, float* const* u, const int32_t* ct) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    if (ct[i] != SOLID) continue;
    int c[3];
    coords(g, i, c);
    for (int k = 0; k < dim; ++k) {
      const G f = faces(g, k);
      u[k][f.at(c[0], c[1], c[2])] = 0.0f;
      u[k][f.at(c[0] + (k == 0), c[1] + (k == 1), c[2] + (k == 2))] = 0.0f;
    }
  }
}

// FluidSimulator.add_gravity (fluid_simulator.py:160-166).
void ors_add_gravity(int dim, const int* res, float* const* u, const double* grav, float dt) {
  const G g = make(dim, res);
  for (int k = 0; k < dim; ++k) {
    if (grav[k] == 0.0) continue;
    const G f = faces(g, k);
    const float gdt = (float)grav[k] * dt;
    for (int64_t i = 0; i < f.cells(); ++i) u[k][i] = u[k][i] + gdt;
  }
}

// update_magnetic_susceptibility: chi = k (1 - theta(phi)).
void ors_update_chi(int dim, const int* res, const float* phi, double k, double eps, float* chi) {
  const G g = make(dim, res);
  const Eps e = eps_consts(eps);
  const float fk = (float)k;
  for (int64_t i = 0; i < g.cells(); ++i) chi[i] = fk * (1.0f - theta(phi[i], e));
}

// update_magnetic_field for axis k: H_k (faces) = H_ext_k - d psi / dx inside.
void ors_update_H(int dim, const int* res, int k, const float* psi, const float* Hext, float dx, float* H) {
  const G g = make(dim, res);
  const G f = faces(g, k);
  for (int64_t i = 0; i < f.cells(); ++i) {
    int c[3];
    coords(f, i, c);
    float h = 0.0f;
    if (c[k] - 1 >= 0 && c[k] < g.n[k]) {
      int cm[3] = {c[0], c[1], c[2]};
      cm[k] -= 1;
      h -= (psi[g.at(c[0], c[1], c[2])] - psi[g.at(cm[0], cm[1], cm[2])]) / dx;
    }
    H[i] = h + Hext[i];
  }
}

// SurfaceTension.calc_n for axis d: n as dim planes of the cell grid.
void ors_calc_n(int dim, const int* res, int d, const float* phi, float dx, float* n) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    float v[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < dim; ++k) {
      float pp[3], pm[3];
      for (int a = 0; a < 3; ++a) {
        const float off = (a == d || a >= dim) ? 0.0f : 0.5f;
        pp[a] = ((float)c[a] + (a == k ? 0.5f : 0.0f)) + off;
        pm[a] = ((float)c[a] - (a == k ? 0.5f : 0.0f)) + off;
      }
      v[k] = (sample(phi, g, pp) - sample(phi, g, pm)) / dx;
    }
    float nn = v[0] * v[0];
    for (int k = 1; k < dim; ++k) nn = nn + v[k] * v[k];
    const float norm = std::sqrt(nn);
    for (int k = 0; k < dim; ++k) n[k * g.cells() + i] = norm > 0.0f ? v[k] / norm : v[k];
  }
}

void ors_calc_kappa(int dim, const int* res, const float* n, float dx, float* kappa) {
  const G g = make(dim, res);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    float acc = 0.0f;
    for (int k = 0; k < dim; ++k) {
      float pp[3], pm[3];
      for (int a = 0; a < 3; ++a) {
        pp[a] = (float)c[a] + (a == k ? 0.5f : 0.0f);
        pm[a] = (float)c[a] - (a == k ? 0.5f : 0.0f);
      }
      const float* nk = n + k * g.cells();
      acc = acc + (sample(nk, g, pp) - sample(nk, g, pm)) / dx;
    }
    kappa[i] = acc;
  }
}

void ors_build_st_b(int dim, const int* res, int d, const float* u, const float* phi, const float* n,
                    const float* kappa, double sigma, double dt, double dx, double eps, float* b) {
  const G g = make(dim, res);
  const G f = faces(g, d);
  const Eps e = eps_consts(eps);
  const float fs = (float)sigma, fdt = (float)dt, fdx = (float)dx, fdx2 = (float)(dx * dx);
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    float bi = u[f.at(c[0], c[1], c[2])] / fdt;
    float pos[3];
    for (int a = 0; a < 3; ++a) pos[a] = (float)c[a] + ((a == d || a >= dim) ? 0.0f : 0.5f);
    const float scale = fs * delta(sample(phi, g, pos), e);
    float nv[3];
    for (int k = 0; k < dim; ++k) nv[k] = n[k * g.cells() + i];
    float du = 0.0f;
    for (int k = 0; k < dim; ++k) {
      float pp[3], pm[3];
      for (int a = 0; a < 3; ++a) {
        pp[a] = (float)c[a] + (a == k ? 0.5f : 0.0f);
        pm[a] = (float)c[a] - (a == k ? 0.5f : 0.0f);
      }
      const float gk = 0.0f + (sample(u, f, pp) - sample(u, f, pm)) / fdx;
      du = k == 0 ? gk * nv[0] : du + gk * nv[k];
    }
    float D2[3][3];
    for (int k1 = 0; k1 < dim; ++k1)
      for (int k2 = 0; k2 < dim; ++k2) {
        float q00[3], q10[3], q01[3], q11[3];
        for (int a = 0; a < 3; ++a) {
          const float h1 = a == k1 ? 0.5f : 0.0f, h2v = a == k2 ? 0.5f : 0.0f, ca = (float)c[a];
          q00[a] = (ca - h1) - h2v;
          q10[a] = (ca + h1) - h2v;
          q01[a] = (ca - h1) + h2v;
          q11[a] = (ca + h1) + h2v;
        }
        const float v00 = sample(u, f, q00), v10 = sample(u, f, q10);
        const float v01 = sample(u, f, q01), v11 = sample(u, f, q11);
        D2[k1][k2] = (v11 + v00 - v10 - v01) / fdx2;
      }
    float d2 = 0.0f;
    for (int j = 0; j < dim; ++j) {
      float t = nv[0] * D2[0][j];
      for (int k = 1; k < dim; ++k) t = t + nv[k] * D2[k][j];
      d2 = j == 0 ? t * nv[0] : d2 + t * nv[j];
    }
    b[i] = bi - scale * (kappa[i] * nv[d] + fdt * (d2 + kappa[i] * du));
  }
}

// One level of the surface tension operator (Adiag, Ax written in full).
void ors_build_st_A(int dim, const int* res, int level, int d, const float* phi, double sigma, double dt,
                    double dx, double eps, float* Adiag, float* Ax) {
  const G fine = make(dim, res);
  int rl[3] = {res[0] >> level, res[1] >> level, dim == 3 ? res[2] >> level : 1};
  const G g = make(dim, rl);
  const Eps e = eps_consts(eps);
  const double dxl = dx * (double)(1 << level);
  const float scale = (float)(sigma * dt / (dxl * dxl)), inv_dt = (float)(1.0 / dt), m = (float)(1 << level);
  for (int64_t i = 0; i < g.cells(); ++i) Adiag[i] = inv_dt;
  for (int64_t i = 0; i < g.cells(); ++i) {
    int c[3];
    coords(g, i, c);
    for (int k = 0; k < dim; ++k) {
      for (int s = 1; s >= -1; s -= 2) {
        if (s > 0 && !(c[k] + 1 < res[k])) continue;
        if (s < 0 && !(c[k] - 1 >= 0)) continue;
        float pos[3];
        for (int a = 0; a < 3; ++a) {
          const float off = (a == d || a >= dim) ? 0.0f : 0.5f;
          pos[a] = (((float)c[a] + (a == k ? 0.5f * (float)s : 0.0f)) + off) * m;
        }
        const float dl = delta(sample(phi, fine, pos), e);
        if (s > 0) Ax[k * g.cells() + i] = -scale * dl;
        Adiag[i] += scale * dl;
      }
    }
  }
}

}  // extern "C"

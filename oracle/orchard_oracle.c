/*
 * Plain-C restatement of the Orchard Flow projection time step (CPU oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests, __graft_entry__.smoke() and the
 * bench's cpu_baseline leg use this library as the checker.  The product path
 * (solver_b200) never links or calls it.
 *
 * Every function restates the reference algorithm in the reference's operation
 * order (sequential loops k-j-i, same association of sums and products, no FMA
 * contraction: built with -ffp-contract=off) so that it reproduces the
 * reference's deterministic CPU build bit for bit; tests/test_oracle.py pins it
 * against oracle/_ref (the reference compiled from source) and against the
 * committed golden fixtures.  Citations are file:line inside the reference
 * project (zfifteen/solver).
 */
#include "orchard_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* errors                                                                   */
/* ------------------------------------------------------------------------ */

static char g_error[512];
enum { OK = 0, EINVAL_ = 1, ERUNTIME = 2 };

static int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
  return code;
}

const char* oo_last_error(void) { return g_error; }

/* ------------------------------------------------------------------------ */
/* layout (core/field_layout.hpp:69-290)                                     */
/* ------------------------------------------------------------------------ */

enum { LOC_CELL = 0, LOC_FX = 1, LOC_FY = 2, LOC_FZ = 3 };
enum { AX = 0, AY = 1, AZ = 2 };

typedef struct {
  int n[3];  /* active extent per axis */
  int s[3];  /* storage extent per axis (active + 2 ghosts) */
  int loc;
  double h[3];
} lay_t;

static lay_t layout_of(const oo_grid* g, int loc) {
  lay_t L;
  L.n[0] = g->nx + (loc == LOC_FX);
  L.n[1] = g->ny + (loc == LOC_FY);
  L.n[2] = g->nz + (loc == LOC_FZ);
  for(int a = 0; a < 3; ++a) L.s[a] = L.n[a] + 2;
  L.loc = loc;
  L.h[0] = g->dx;
  L.h[1] = g->dy;
  L.h[2] = g->dz;
  return L;
}

static size_t lay_size(const lay_t* L) { return (size_t)L->s[0] * L->s[1] * L->s[2]; }

/* index i + sx*j + sx*sy*k (core/field_layout.hpp:178-183) */
#define IDX(L, i, j, k) \
  ((size_t)(i) + (size_t)(L)->s[0] * (size_t)(j) + (size_t)(L)->s[0] * (size_t)(L)->s[1] * (size_t)(k))

typedef struct {
  int b[3], e[3]; /* [begin, end) per axis */
} range_t;

static range_t active_range(const lay_t* L) {
  range_t r;
  for(int a = 0; a < 3; ++a) {
    r.b[a] = 1;
    r.e[a] = 1 + L->n[a];
  }
  return r;
}

/* face index: 0 x_min, 1 x_max, 2 y_min, 3 y_max, 4 z_min, 5 z_max */
static int face_axis(int face) { return face / 2; }
static int face_is_lower(int face) { return (face % 2) == 0; }

static range_t boundary_active_range(const lay_t* L, int face) {
  range_t r = active_range(L);
  int a = face_axis(face);
  int first = face_is_lower(face) ? 1 : 1 + L->n[a] - 1;
  r.b[a] = first;
  r.e[a] = first + 1;
  return r;
}

static range_t ghost_range(const lay_t* L, int face) {
  range_t r = active_range(L);
  int a = face_axis(face);
  int begin = face_is_lower(face) ? 0 : 1 + L->n[a];
  r.b[a] = begin;
  r.e[a] = begin + 1;
  return r;
}

static double* alloc_field(const lay_t* L) { return (double*)calloc(lay_size(L), sizeof(double)); }
static double* clone_field(const lay_t* L, const double* src) {
  double* f = (double*)malloc(lay_size(L) * sizeof(double));
  memcpy(f, src, lay_size(L) * sizeof(double));
  return f;
}
static void copy_field(const lay_t* L, double* dst, const double* src) {
  memcpy(dst, src, lay_size(L) * sizeof(double));
}

/* copy_range (solver/projection.cpp:90-110) */
static void copy_range(const lay_t* L, double* dst, range_t dr, const double* src, range_t sr) {
  int ex = dr.e[0] - dr.b[0], ey = dr.e[1] - dr.b[1], ez = dr.e[2] - dr.b[2];
  for(int k = 0; k < ez; ++k)
    for(int j = 0; j < ey; ++j)
      for(int i = 0; i < ex; ++i)
        dst[IDX(L, dr.b[0] + i, dr.b[1] + j, dr.b[2] + k)] =
            src[IDX(L, sr.b[0] + i, sr.b[1] + j, sr.b[2] + k)];
}

#define FOR_ACTIVE(L)                                  \
  for(int k = 1; k < 1 + (L)->n[2]; ++k)               \
    for(int j = 1; j < 1 + (L)->n[1]; ++j)             \
      for(int i = 1; i < 1 + (L)->n[0]; ++i)

static double active_mean(const lay_t* L, const double* f) {
  double sum = 0.0;
  size_t count = (size_t)L->n[0] * L->n[1] * L->n[2];
  FOR_ACTIVE(L) sum += f[IDX(L, i, j, k)];
  return sum / (double)count;
}

static double subtract_active_mean(const lay_t* L, double* f) {
  double mean = active_mean(L, f);
  FOR_ACTIVE(L) f[IDX(L, i, j, k)] -= mean;
  return mean;
}

static double active_l2_norm(const lay_t* L, const double* f) {
  double sum = 0.0;
  size_t count = (size_t)L->n[0] * L->n[1] * L->n[2];
  FOR_ACTIVE(L) sum += f[IDX(L, i, j, k)] * f[IDX(L, i, j, k)];
  return sqrt(sum / (double)count);
}

static double dot_active(const lay_t* L, const double* a, const double* b) {
  double sum = 0.0;
  FOR_ACTIVE(L) sum += a[IDX(L, i, j, k)] * b[IDX(L, i, j, k)];
  return sum;
}

static void axpy_active(const lay_t* L, double* dst, const double* src, double scale) {
  FOR_ACTIVE(L) dst[IDX(L, i, j, k)] += scale * src[IDX(L, i, j, k)];
}

static void scale_active(const lay_t* L, double* f, double scale) {
  FOR_ACTIVE(L) f[IDX(L, i, j, k)] *= scale;
}

static void copy_active(const lay_t* L, double* dst, const double* src) {
  FOR_ACTIVE(L) dst[IDX(L, i, j, k)] = src[IDX(L, i, j, k)];
}

static void fill_storage(const lay_t* L, double* f, double v) {
  size_t n = lay_size(L);
  for(size_t q = 0; q < n; ++q) f[q] = v;
}

/* ------------------------------------------------------------------------ */
/* validation helpers                                                       */
/* ------------------------------------------------------------------------ */

static int check_grid(const oo_grid* g) {
  if(g->nx <= 0 || g->ny <= 0 || g->nz <= 0)
    return fail(EINVAL_, "grid dimensions must be positive");
  if(g->dx <= 0.0 || g->dy <= 0.0 || g->dz <= 0.0)
    return fail(EINVAL_, "grid spacing must be positive");
  return OK;
}

/* ------------------------------------------------------------------------ */
/* discrete operators (operators/discrete_operators.cpp:24-123)              */
/* ------------------------------------------------------------------------ */

static double second_derivative(const lay_t* L, const double* f, int i, int j, int k, int axis) {
  double spacing = L->h[axis];
  double inv = 1.0 / (spacing * spacing);
  switch(axis) {
    case AX:
      return (f[IDX(L, i + 1, j, k)] - 2.0 * f[IDX(L, i, j, k)] + f[IDX(L, i - 1, j, k)]) * inv;
    case AY:
      return (f[IDX(L, i, j + 1, k)] - 2.0 * f[IDX(L, i, j, k)] + f[IDX(L, i, j - 1, k)]) * inv;
    default:
      return (f[IDX(L, i, j, k + 1)] - 2.0 * f[IDX(L, i, j, k)] + f[IDX(L, i, j, k - 1)]) * inv;
  }
}

/* compute_component_laplacian (operators/discrete_operators.cpp:47-60) */
static void laplacian_component(const lay_t* L, const double* in, double* out) {
  FOR_ACTIVE(L) {
    out[IDX(L, i, j, k)] = second_derivative(L, in, i, j, k, AX) +
                           second_derivative(L, in, i, j, k, AY) +
                           second_derivative(L, in, i, j, k, AZ);
  }
}

/* compute_gradient (operators/discrete_operators.cpp:64-96) */
static void gradient(const oo_grid* g, const double* p, double* gu, double* gv, double* gw) {
  lay_t P = layout_of(g, LOC_CELL);
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  FOR_ACTIVE(&U) gu[IDX(&U, i, j, k)] = (p[IDX(&P, i, j, k)] - p[IDX(&P, i - 1, j, k)]) / g->dx;
  FOR_ACTIVE(&V) gv[IDX(&V, i, j, k)] = (p[IDX(&P, i, j, k)] - p[IDX(&P, i, j - 1, k)]) / g->dy;
  FOR_ACTIVE(&W) gw[IDX(&W, i, j, k)] = (p[IDX(&P, i, j, k)] - p[IDX(&P, i, j, k - 1)]) / g->dz;
}

/* compute_divergence (operators/discrete_operators.cpp:98-113) */
static void divergence(const oo_grid* g, const double* u, const double* v, const double* w,
                       double* div) {
  lay_t P = layout_of(g, LOC_CELL);
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  FOR_ACTIVE(&P) {
    double du = (u[IDX(&U, i + 1, j, k)] - u[IDX(&U, i, j, k)]) / g->dx;
    double dv = (v[IDX(&V, i, j + 1, k)] - v[IDX(&V, i, j, k)]) / g->dy;
    double dw = (w[IDX(&W, i, j, k + 1)] - w[IDX(&W, i, j, k)]) / g->dz;
    div[IDX(&P, i, j, k)] = du + dv + dw;
  }
}

/* ------------------------------------------------------------------------ */
/* momentum terms (solver/momentum_terms.cpp)                                */
/* ------------------------------------------------------------------------ */

static const double kSmallDenominator = 1.0e-14;

/* limiter_value, van Leer (solver/momentum_terms.cpp:26-33) */
static double van_leer(double r) { return (r + fabs(r)) / (1.0 + fabs(r)); }

/* safe_ratio (solver/momentum_terms.cpp:35-40) */
static double safe_ratio(double num, double den) {
  if(fabs(den) < kSmallDenominator) return 0.0;
  return num / den;
}

/* reconstruct_face_{x,y,z} (solver/momentum_terms.cpp:42-151), TVD scheme.
 * The axis-generic form: q(o) reads the field at offset o along `axis` from
 * the face's right/upper cell; `right_index` is that cell's storage index
 * along the axis and `max_index` the last storage index. */
static double reconstruct(const lay_t* L, const double* f, int i, int j, int k, int axis,
                          double face_velocity) {
  int di = axis == AX, dj = axis == AY, dk = axis == AZ;
  double left = f[IDX(L, i - di, j - dj, k - dk)];
  double right = f[IDX(L, i, j, k)];
  if(fabs(face_velocity) < kSmallDenominator) return face_velocity >= 0.0 ? left : right;
  int right_index = axis == AX ? i : axis == AY ? j : k;
  int max_index = L->s[axis] - 1;
  if(face_velocity >= 0.0) {
    if(right_index - 2 < 0) return left;
    double delta_down = right - left;
    double ratio = safe_ratio(left - f[IDX(L, i - 2 * di, j - 2 * dj, k - 2 * dk)], delta_down);
    return left + 0.5 * van_leer(ratio) * delta_down;
  }
  if(right_index + 1 > max_index) return right;
  double delta = right - left;
  double ratio = safe_ratio(f[IDX(L, i + di, j + dj, k + dk)] - right, delta);
  return right - 0.5 * van_leer(ratio) * delta;
}

/* compute_{u,v,w}_advection (solver/momentum_terms.cpp:153-266) */
static void advection_component(const oo_grid* g, int comp, const double* u, const double* v,
                                const double* w, double* out) {
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  const lay_t* C = comp == 0 ? &U : comp == 1 ? &V : &W;
  const double* f = comp == 0 ? u : comp == 1 ? v : w;
  FOR_ACTIVE(C) {
    double wv, ev, sv, nv, bv, fv;
    if(comp == 0) {
      wv = 0.5 * (u[IDX(&U, i - 1, j, k)] + u[IDX(&U, i, j, k)]);
      ev = 0.5 * (u[IDX(&U, i, j, k)] + u[IDX(&U, i + 1, j, k)]);
      sv = 0.5 * (v[IDX(&V, i - 1, j, k)] + v[IDX(&V, i, j, k)]);
      nv = 0.5 * (v[IDX(&V, i - 1, j + 1, k)] + v[IDX(&V, i, j + 1, k)]);
      bv = 0.5 * (w[IDX(&W, i - 1, j, k)] + w[IDX(&W, i, j, k)]);
      fv = 0.5 * (w[IDX(&W, i - 1, j, k + 1)] + w[IDX(&W, i, j, k + 1)]);
    } else if(comp == 1) {
      wv = 0.5 * (u[IDX(&U, i, j - 1, k)] + u[IDX(&U, i, j, k)]);
      ev = 0.5 * (u[IDX(&U, i + 1, j - 1, k)] + u[IDX(&U, i + 1, j, k)]);
      sv = 0.5 * (v[IDX(&V, i, j - 1, k)] + v[IDX(&V, i, j, k)]);
      nv = 0.5 * (v[IDX(&V, i, j, k)] + v[IDX(&V, i, j + 1, k)]);
      bv = 0.5 * (w[IDX(&W, i, j - 1, k)] + w[IDX(&W, i, j, k)]);
      fv = 0.5 * (w[IDX(&W, i, j - 1, k + 1)] + w[IDX(&W, i, j, k + 1)]);
    } else {
      wv = 0.5 * (u[IDX(&U, i, j, k - 1)] + u[IDX(&U, i, j, k)]);
      ev = 0.5 * (u[IDX(&U, i + 1, j, k - 1)] + u[IDX(&U, i + 1, j, k)]);
      sv = 0.5 * (v[IDX(&V, i, j, k - 1)] + v[IDX(&V, i, j, k)]);
      nv = 0.5 * (v[IDX(&V, i, j + 1, k - 1)] + v[IDX(&V, i, j + 1, k)]);
      bv = 0.5 * (w[IDX(&W, i, j, k - 1)] + w[IDX(&W, i, j, k)]);
      fv = 0.5 * (w[IDX(&W, i, j, k)] + w[IDX(&W, i, j, k + 1)]);
    }
    double west = wv * reconstruct(C, f, i, j, k, AX, wv);
    double east = ev * reconstruct(C, f, i + 1, j, k, AX, ev);
    double south = sv * reconstruct(C, f, i, j, k, AY, sv);
    double north = nv * reconstruct(C, f, i, j + 1, k, AY, nv);
    double back = bv * reconstruct(C, f, i, j, k, AZ, bv);
    double front = fv * reconstruct(C, f, i, j, k + 1, AZ, fv);
    out[IDX(C, i, j, k)] = (east - west) / g->dx + (north - south) / g->dy + (front - back) / g->dz;
  }
}

static void advection(const oo_grid* g, const double* u, const double* v, const double* w,
                      double* au, double* av, double* aw) {
  advection_component(g, 0, u, v, w, au);
  advection_component(g, 1, u, v, w, av);
  advection_component(g, 2, u, v, w, aw);
}

/* compute_diffusion_term (solver/momentum_terms.cpp:316-325) */
static void diffusion(const oo_grid* g, double nu, const double* u, const double* v,
                      const double* w, double* du, double* dv, double* dw) {
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  laplacian_component(&U, u, du);
  laplacian_component(&V, v, dv);
  laplacian_component(&W, w, dw);
  scale_active(&U, du, nu);
  scale_active(&V, dv, nu);
  scale_active(&W, dw, nu);
}

/* compute_advective_cfl (solver/momentum_terms.cpp:327-355) */
static double advective_cfl(const oo_grid* g, const double* u, const double* v, const double* w,
                            double dt) {
  lay_t P = layout_of(g, LOC_CELL);
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  double max_cfl = 0.0;
  FOR_ACTIVE(&P) {
    double uc = 0.5 * (u[IDX(&U, i, j, k)] + u[IDX(&U, i + 1, j, k)]);
    double vc = 0.5 * (v[IDX(&V, i, j, k)] + v[IDX(&V, i, j + 1, k)]);
    double wc = 0.5 * (w[IDX(&W, i, j, k)] + w[IDX(&W, i, j, k + 1)]);
    double local = dt * (fabs(uc) / g->dx + fabs(vc) / g->dy + fabs(wc) / g->dz);
    if(local > max_cfl) max_cfl = local;
  }
  return max_cfl;
}

/* ------------------------------------------------------------------------ */
/* boundary conditions (solver/projection.cpp:45-80, 187-462, 934-1026)      */
/* ------------------------------------------------------------------------ */

static int is_dirichlet_velocity(int type) {
  return type == OO_NO_SLIP_WALL || type == OO_PRESCRIBED_VELOCITY || type == OO_SYMMETRY;
}

static int velocity_axis_periodic(const oo_bc* bc, int axis, int* periodic) {
  int lo = bc->faces[2 * axis].type == OO_PERIODIC;
  int hi = bc->faces[2 * axis + 1].type == OO_PERIODIC;
  if(lo != hi) return fail(EINVAL_, "periodic velocity boundaries must be paired on both sides");
  *periodic = lo;
  return OK;
}

static int pressure_axis_periodic(const oo_pbc* bc, int axis, int* periodic) {
  int lo = bc->faces[2 * axis].type == OO_P_PERIODIC;
  int hi = bc->faces[2 * axis + 1].type == OO_P_PERIODIC;
  if(lo != hi) return fail(EINVAL_, "periodic pressure boundaries must be paired on both sides");
  *periodic = lo;
  return OK;
}

/* apply_periodic_pair, non-duplicated axis (solver/projection.cpp:207-231) */
static void periodic_pair_plain(const lay_t* L, double* f, int axis) {
  range_t act = active_range(L);
  range_t src_lo = act, src_hi = act;
  src_lo.b[axis] = act.e[axis] - 1;
  src_hi.e[axis] = act.b[axis] + 1;
  copy_range(L, f, ghost_range(L, 2 * axis), f, src_lo);
  copy_range(L, f, ghost_range(L, 2 * axis + 1), f, src_hi);
}

/* apply_periodic_pair for a face field (solver/projection.cpp:233-300) */
static void periodic_pair_face(const lay_t* L, int normal, double* f, int axis) {
  if(normal == axis) {
    range_t lb = boundary_active_range(L, 2 * axis), ub = boundary_active_range(L, 2 * axis + 1);
    int ex = lb.e[0] - lb.b[0], ey = lb.e[1] - lb.b[1], ez = lb.e[2] - lb.b[2];
    for(int k = 0; k < ez; ++k)
      for(int j = 0; j < ey; ++j)
        for(int i = 0; i < ex; ++i) {
          size_t a = IDX(L, lb.b[0] + i, lb.b[1] + j, lb.b[2] + k);
          size_t b = IDX(L, ub.b[0] + i, ub.b[1] + j, ub.b[2] + k);
          double shared = 0.5 * (f[a] + f[b]);
          f[a] = shared;
          f[b] = shared;
        }
    range_t act = active_range(L);
    range_t src_lo = act, src_hi = act;
    src_lo.b[axis] = act.e[axis] - 2;
    src_lo.e[axis] = act.e[axis] - 1;
    src_hi.b[axis] = act.b[axis] + 1;
    src_hi.e[axis] = act.b[axis] + 2;
    copy_range(L, f, ghost_range(L, 2 * axis), f, src_lo);
    copy_range(L, f, ghost_range(L, 2 * axis + 1), f, src_hi);
    return;
  }
  periodic_pair_plain(L, f, axis);
}

/* apply_face_field_boundary (solver/projection.cpp:384-449) */
static void face_field_boundary(const lay_t* L, int comp, double* f, int face,
                                const oo_face_bc* c) {
  if(c->type == OO_PERIODIC) return;
  int baxis = face_axis(face);
  int lower = face_is_lower(face);
  range_t ba = boundary_active_range(L, face), gr = ghost_range(L, face);
  int ex = ba.e[0] - ba.b[0], ey = ba.e[1] - ba.b[1], ez = ba.e[2] - ba.b[2];
  for(int k = 0; k < ez; ++k)
    for(int j = 0; j < ey; ++j)
      for(int i = 0; i < ex; ++i) {
        int bi = ba.b[0] + i, bj = ba.b[1] + j, bk = ba.b[2] + k;
        int gi = gr.b[0] + i, gj = gr.b[1] + j, gk = gr.b[2] + k;
        if(comp == baxis) {
          int s = lower ? 1 : -1;
          int ii = bi + s * (baxis == AX), jj = bj + s * (baxis == AY), kk = bk + s * (baxis == AZ);
          if(c->type == OO_FIXED_PRESSURE) {
            f[IDX(L, bi, bj, bk)] = f[IDX(L, ii, jj, kk)];
            f[IDX(L, gi, gj, gk)] = f[IDX(L, bi, bj, bk)];
            continue;
          }
          double bv = c->type == OO_SYMMETRY ? 0.0 : c->velocity[comp];
          f[IDX(L, bi, bj, bk)] = bv;
          f[IDX(L, gi, gj, gk)] = 2.0 * bv - f[IDX(L, ii, jj, kk)];
          continue;
        }
        if(c->type == OO_NO_SLIP_WALL || c->type == OO_PRESCRIBED_VELOCITY) {
          double wall = c->velocity[comp];
          f[IDX(L, gi, gj, gk)] = 2.0 * wall - f[IDX(L, bi, bj, bk)];
        } else if(c->type == OO_SYMMETRY || c->type == OO_FIXED_PRESSURE) {
          f[IDX(L, gi, gj, gk)] = f[IDX(L, bi, bj, bk)];
        }
      }
}

/* apply_velocity_component_boundaries (solver/projection.cpp:451-462) */
static int component_boundaries(const oo_grid* g, const oo_bc* bc, int comp, double* f) {
  lay_t L = layout_of(g, LOC_FX + comp);
  for(int axis = 0; axis < 3; ++axis) {
    int periodic = 0;
    int rc = velocity_axis_periodic(bc, axis, &periodic);
    if(rc) return rc;
    if(periodic) {
      periodic_pair_face(&L, comp, f, axis);
      continue;
    }
    face_field_boundary(&L, comp, f, 2 * axis, &bc->faces[2 * axis]);
    face_field_boundary(&L, comp, f, 2 * axis + 1, &bc->faces[2 * axis + 1]);
  }
  return OK;
}

static int velocity_bc(const oo_grid* g, const oo_bc* bc, double* u, double* v, double* w) {
  int rc = component_boundaries(g, bc, 0, u);
  if(!rc) rc = component_boundaries(g, bc, 1, v);
  if(!rc) rc = component_boundaries(g, bc, 2, w);
  return rc;
}

/* apply_pressure_face_boundary (solver/projection.cpp:302-337) */
static void pressure_face_boundary(const lay_t* L, double* p, int face, int type, double value,
                                   double grad) {
  int axis = face_axis(face);
  range_t ba = boundary_active_range(L, face), gr = ghost_range(L, face);
  double spacing = L->h[axis];
  int ex = ba.e[0] - ba.b[0], ey = ba.e[1] - ba.b[1], ez = ba.e[2] - ba.b[2];
  for(int k = 0; k < ez; ++k)
    for(int j = 0; j < ey; ++j)
      for(int i = 0; i < ex; ++i) {
        double av = p[IDX(L, ba.b[0] + i, ba.b[1] + j, ba.b[2] + k)];
        size_t gq = IDX(L, gr.b[0] + i, gr.b[1] + j, gr.b[2] + k);
        if(type == OO_P_NEUMANN)
          p[gq] = face_is_lower(face) ? av - grad * spacing : av + grad * spacing;
        else if(type == OO_P_DIRICHLET)
          p[gq] = 2.0 * value - av;
      }
}

static int pressure_bc(const oo_grid* g, const oo_pbc* pbc, double* p) {
  lay_t L = layout_of(g, LOC_CELL);
  for(int axis = 0; axis < 3; ++axis) {
    int periodic = 0;
    int rc = pressure_axis_periodic(pbc, axis, &periodic);
    if(rc) return rc;
    if(periodic) {
      periodic_pair_plain(&L, p, axis);
      continue;
    }
    for(int s = 0; s < 2; ++s) {
      const oo_pface_bc* c = &pbc->faces[2 * axis + s];
      pressure_face_boundary(&L, p, 2 * axis + s, c->type, c->value, c->gradient);
    }
  }
  return OK;
}

/* derive_pressure_correction_boundary_conditions (solver/projection.cpp:934-964) */
static int derive_pbc(const oo_bc* bc, oo_pbc* out) {
  memset(out, 0, sizeof(*out));
  for(int f = 0; f < 6; ++f) {
    switch(bc->faces[f].type) {
      case OO_NO_SLIP_WALL:
      case OO_PRESCRIBED_VELOCITY:
      case OO_SYMMETRY:
        out->faces[f].type = OO_P_NEUMANN;
        out->faces[f].gradient = 0.0;
        break;
      case OO_FIXED_PRESSURE:
        out->faces[f].type = OO_P_DIRICHLET;
        out->faces[f].value = 0.0;
        break;
      default:
        out->faces[f].type = OO_P_PERIODIC;
        break;
    }
  }
  for(int axis = 0; axis < 3; ++axis) {
    int periodic = 0;
    int rc = pressure_axis_periodic(out, axis, &periodic);
    if(rc) return rc;
  }
  return OK;
}

/* apply_total_pressure_gradient_face (solver/projection.cpp:339-382) */
static void total_pressure_gradient_face(const oo_grid* g, double* p, int face, const double* src,
                                         int comp) {
  lay_t P = layout_of(g, LOC_CELL);
  lay_t S = layout_of(g, LOC_FX + comp);
  int axis = face_axis(face);
  int lower = face_is_lower(face);
  range_t ba = boundary_active_range(&P, face), gr = ghost_range(&P, face);
  range_t wa = active_range(&S);
  double spacing = P.h[axis];
  int ex = ba.e[0] - ba.b[0], ey = ba.e[1] - ba.b[1], ez = ba.e[2] - ba.b[2];
  for(int k = 0; k < ez; ++k)
    for(int j = 0; j < ey; ++j)
      for(int i = 0; i < ex; ++i) {
        int bi = ba.b[0] + i, bj = ba.b[1] + j, bk = ba.b[2] + k;
        int w[3] = {bi, bj, bk};
        w[axis] = lower ? wa.b[axis] : wa.e[axis] - 1;
        double gradv = src[IDX(&S, w[0], w[1], w[2])];
        double av = p[IDX(&P, bi, bj, bk)];
        p[IDX(&P, gr.b[0] + i, gr.b[1] + j, gr.b[2] + k)] =
            lower ? av - gradv * spacing : av + gradv * spacing;
      }
}

/* apply_total_pressure_boundary_conditions (solver/projection.cpp:986-1026) */
static int total_pressure_bc(const oo_grid* g, const oo_bc* bc, const double* su,
                             const double* sv, const double* sw, double* p) {
  lay_t P = layout_of(g, LOC_CELL);
  const double* src[3] = {su, sv, sw};
  for(int axis = 0; axis < 3; ++axis) {
    int periodic = 0;
    int rc = velocity_axis_periodic(bc, axis, &periodic);
    if(rc) return rc;
    if(periodic) {
      periodic_pair_plain(&P, p, axis);
      continue;
    }
    for(int s = 0; s < 2; ++s) {
      int face = 2 * axis + s;
      const oo_face_bc* c = &bc->faces[face];
      switch(c->type) {
        case OO_NO_SLIP_WALL:
        case OO_PRESCRIBED_VELOCITY:
        case OO_SYMMETRY:
          total_pressure_gradient_face(g, p, face, src[axis], axis);
          break;
        case OO_FIXED_PRESSURE:
          pressure_face_boundary(&P, p, face, OO_P_DIRICHLET, c->pressure, 0.0);
          break;
        default:
          break;
      }
    }
  }
  return OK;
}

/* ------------------------------------------------------------------------ */
/* ADI predictor (solver/projection.cpp:464-888, 1028-1047)                  */
/* ------------------------------------------------------------------------ */

static const double kSmallNumber = 1.0e-30;

/* solve_tridiagonal, Thomas (solver/projection.cpp:522-559) */
static int thomas(int n, const double* lo, const double* di, const double* up, const double* rhs,
                  double* sol, double* mu, double* mr) {
  if(n == 0) return OK;
  double pivot = di[0];
  if(fabs(pivot) < kSmallNumber) return fail(ERUNTIME, "tridiagonal solve encountered a zero pivot");
  mu[0] = n > 1 ? up[0] / pivot : 0.0;
  mr[0] = rhs[0] / pivot;
  for(int i = 1; i < n; ++i) {
    pivot = di[i] - lo[i] * mu[i - 1];
    if(fabs(pivot) < kSmallNumber)
      return fail(ERUNTIME, "tridiagonal solve encountered a zero pivot");
    mu[i] = i + 1 < n ? up[i] / pivot : 0.0;
    mr[i] = (rhs[i] - lo[i] * mr[i - 1]) / pivot;
  }
  sol[n - 1] = mr[n - 1];
  for(int i = n - 1; i-- > 0;) sol[i] = mr[i] - mu[i] * sol[i + 1];
  return OK;
}

typedef struct {
  double *lo, *di, *up, *rhs, *sol, *mu, *mr, *dm, *lm, *um, *x, *u, *z;
} tri_work;

static tri_work tri_alloc(int n) {
  tri_work t;
  double* base = (double*)calloc((size_t)13 * (n > 0 ? n : 1), sizeof(double));
  double** p[13] = {&t.lo, &t.di, &t.up, &t.rhs, &t.sol, &t.mu, &t.mr,
                    &t.dm, &t.lm, &t.um, &t.x, &t.u, &t.z};
  for(int q = 0; q < 13; ++q) *p[q] = base + (size_t)q * (n > 0 ? n : 1);
  return t;
}
static void tri_free(tri_work* t) { free(t->lo); }

/* solve_cyclic_tridiagonal, Sherman-Morrison (solver/projection.cpp:561-617) */
static int cyclic_thomas(int n, tri_work* t, double lower_corner, double upper_corner) {
  if(n == 0) return OK;
  if(n == 1) {
    double pivot = t->di[0] + lower_corner + upper_corner;
    if(fabs(pivot) < kSmallNumber)
      return fail(ERUNTIME, "cyclic tridiagonal solve encountered a zero pivot");
    t->sol[0] = t->rhs[0] / pivot;
    return OK;
  }
  for(int i = 0; i < n; ++i) {
    t->dm[i] = t->di[i];
    t->lm[i] = t->lo[i];
    t->um[i] = t->up[i];
  }
  double gamma = -t->di[0];
  if(fabs(gamma) < kSmallNumber)
    return fail(ERUNTIME, "cyclic tridiagonal solve encountered a zero gamma");
  t->dm[0] = t->di[0] - gamma;
  t->dm[n - 1] = t->di[n - 1] - lower_corner * upper_corner / gamma;
  t->lm[0] = 0.0;
  t->um[n - 1] = 0.0;
  int rc = thomas(n, t->lm, t->dm, t->um, t->rhs, t->x, t->mu, t->mr);
  if(rc) return rc;
  for(int i = 0; i < n; ++i) t->u[i] = 0.0;
  t->u[0] = gamma;
  t->u[n - 1] = lower_corner;
  rc = thomas(n, t->lm, t->dm, t->um, t->u, t->z, t->mu, t->mr);
  if(rc) return rc;
  double denominator = 1.0 + t->z[0] + upper_corner * t->z[n - 1] / gamma;
  if(fabs(denominator) < kSmallNumber)
    return fail(ERUNTIME, "cyclic tridiagonal solve encountered a singular Sherman-Morrison update");
  double factor = (t->x[0] + upper_corner * t->x[n - 1] / gamma) / denominator;
  for(int i = 0; i < n; ++i) t->sol[i] = t->x[i] - factor * t->z[i];
  return OK;
}

/* GhostRelation (solver/projection.cpp:51-80) */
static void tangential_ghost_relation(const oo_face_bc* c, int comp, double* coef, double* cst) {
  switch(c->type) {
    case OO_NO_SLIP_WALL:
    case OO_PRESCRIBED_VELOCITY:
      *coef = -1.0;
      *cst = 2.0 * c->velocity[comp];
      return;
    case OO_SYMMETRY:
    case OO_FIXED_PRESSURE:
      *coef = 1.0;
      *cst = 0.0;
      return;
    default:
      *coef = 0.0;
      *cst = 0.0;
      return;
  }
}

/* The line through (i,j,k) along `axis`: position q of a line-local index. */
static size_t line_pos(const lay_t* L, int axis, int a, int b, int q) {
  /* (a, b) are the two other storage coordinates in the loop order used by
   * the reference: x-lines loop k then j, y-lines k then i, z-lines j then i. */
  switch(axis) {
    case AX: return IDX(L, q, b, a);
    case AY: return IDX(L, b, q, a);
    default: return IDX(L, b, a, q);
  }
}

/* solve_component_sweep_periodic (solver/projection.cpp:619-720) and
 * solve_component_sweep (solver/projection.cpp:722-866) */
static int component_sweep(const oo_grid* g, const oo_bc* bc, int comp, const double* in,
                           int axis, double alpha, double* out, int* line_solves) {
  lay_t L = layout_of(g, LOC_FX + comp);
  range_t act = active_range(&L);
  int periodic = 0;
  int rc = velocity_axis_periodic(bc, axis, &periodic);
  if(rc) return rc;
  double spacing = L.h[axis];
  double beta = alpha / (spacing * spacing);
  int begin, end;
  if(periodic) {
    begin = act.b[axis];
    end = comp == axis ? act.e[axis] - 1 : act.e[axis];
  } else if(comp != axis) {
    begin = act.b[axis];
    end = act.e[axis];
  } else {
    begin = act.b[axis] + (is_dirichlet_velocity(bc->faces[2 * axis].type) ? 1 : 0);
    end = act.e[axis] - (is_dirichlet_velocity(bc->faces[2 * axis + 1].type) ? 1 : 0);
  }
  int n = end - begin;
  if(n <= 0) return OK;
  /* outer loop over the first of the other axes, inner over the second */
  int oa = axis == AX ? AZ : axis == AY ? AZ : AY;  /* outer axis */
  int ia = axis == AX ? AY : AX;                     /* inner axis */
  tri_work t = tri_alloc(n);
  for(int q = 0; q < n; ++q) {
    t.lo[q] = -beta;
    t.di[q] = 1.0 + 2.0 * beta;
    t.up[q] = -beta;
  }
  t.lo[0] = 0.0;
  t.up[n - 1] = 0.0;
  for(int a = act.b[oa]; a < act.e[oa] && !rc; ++a) {
    for(int b = act.b[ia]; b < act.e[ia]; ++b) {
      for(int q = begin; q < end; ++q) t.rhs[q - begin] = in[line_pos(&L, axis, a, b, q)];
      if(periodic) {
        rc = cyclic_thomas(n, &t, -beta, -beta);
        if(rc) break;
        for(int q = begin; q < end; ++q) out[line_pos(&L, axis, a, b, q)] = t.sol[q - begin];
        if(comp == axis)
          out[line_pos(&L, axis, a, b, act.e[axis] - 1)] = out[line_pos(&L, axis, a, b, begin)];
      } else {
        for(int q = 0; q < n; ++q) t.di[q] = 1.0 + 2.0 * beta;
        const oo_face_bc* lo = &bc->faces[2 * axis];
        const oo_face_bc* hi = &bc->faces[2 * axis + 1];
        if(comp == axis && is_dirichlet_velocity(lo->type)) {
          t.rhs[0] += beta * lo->velocity[axis];
        } else {
          double coef, cst;
          tangential_ghost_relation(lo, comp, &coef, &cst);
          t.di[0] -= beta * coef;
          t.rhs[0] += beta * cst;
        }
        if(comp == axis && is_dirichlet_velocity(hi->type)) {
          t.rhs[n - 1] += beta * hi->velocity[axis];
        } else {
          double coef, cst;
          tangential_ghost_relation(hi, comp, &coef, &cst);
          t.di[n - 1] -= beta * coef;
          t.rhs[n - 1] += beta * cst;
        }
        rc = thomas(n, t.lo, t.di, t.up, t.rhs, t.sol, t.mu, t.mr);
        if(rc) break;
        for(int q = begin; q < end; ++q) out[line_pos(&L, axis, a, b, q)] = t.sol[q - begin];
      }
      ++*line_solves;
    }
  }
  tri_free(&t);
  return rc;
}

/* solve_component_adi (solver/projection.cpp:868-888) */
static int component_adi(const oo_grid* g, const oo_bc* bc, int comp, double* field, double alpha,
                         int* line_solves) {
  lay_t L = layout_of(g, LOC_FX + comp);
  int rc = component_boundaries(g, bc, comp, field);
  if(rc || alpha == 0.0) return rc;
  double* working = clone_field(&L, field);
  double* next = alloc_field(&L);
  for(int axis = 0; axis < 3 && !rc; ++axis) {
    copy_field(&L, next, working);
    rc = component_sweep(g, bc, comp, working, axis, alpha, next, line_solves);
    if(!rc) rc = component_boundaries(g, bc, comp, next);
    copy_field(&L, working, next);
  }
  if(!rc) copy_field(&L, field, working);
  free(working);
  free(next);
  return rc;
}

static int predictor_adi(const oo_grid* g, const oo_bc* bc, double alpha, const double* ru,
                         const double* rv, const double* rw, double* pu, double* pv, double* pw,
                         int* line_solves) {
  if(alpha < 0.0) return fail(EINVAL_, "solve_predictor_adi expects a non-negative alpha");
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  copy_field(&U, pu, ru);
  copy_field(&V, pv, rv);
  copy_field(&W, pw, rw);
  int rc = component_adi(g, bc, 0, pu, alpha, line_solves);
  if(!rc) rc = component_adi(g, bc, 1, pv, alpha, line_solves);
  if(!rc) rc = component_adi(g, bc, 2, pw, alpha, line_solves);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* MG-PCG Poisson (linsolve/poisson_solver.cpp)                              */
/* ------------------------------------------------------------------------ */

/* neighbor_value (linsolve/poisson_solver.cpp:195-242) */
static double neighbor_value(const lay_t* L, const double* in, const oo_pbc* bc, int i, int j,
                             int k, int axis, int upper) {
  int c = axis == AX ? i : axis == AY ? j : k;
  int begin = 1, end = 1 + L->n[axis];
  int di = axis == AX, dj = axis == AY, dk = axis == AZ;
  if((!upper && c > begin) || (upper && c < end - 1)) {
    int s = upper ? 1 : -1;
    return in[IDX(L, i + s * di, j + s * dj, k + s * dk)];
  }
  const oo_pface_bc* b = &bc->faces[2 * axis + (upper ? 1 : 0)];
  double center = in[IDX(L, i, j, k)];
  double spacing = L->h[axis];
  switch(b->type) {
    case OO_P_PERIODIC: {
      int t = upper ? begin : end - 1;
      return in[IDX(L, axis == AX ? t : i, axis == AY ? t : j, axis == AZ ? t : k)];
    }
    case OO_P_NEUMANN:
      return upper ? center + b->gradient * spacing : center - b->gradient * spacing;
    case OO_P_DIRICHLET:
      return 2.0 * b->value - center;
  }
  return center;
}

/* apply_poisson_operator (linsolve/poisson_solver.cpp:244-269) */
static void poisson_operator(const lay_t* L, const double* in, const oo_pbc* bc, double* out) {
  double dx = L->h[0], dy = L->h[1], dz = L->h[2];
  FOR_ACTIVE(L) {
    double center = in[IDX(L, i, j, k)];
    double left = neighbor_value(L, in, bc, i, j, k, AX, 0);
    double right = neighbor_value(L, in, bc, i, j, k, AX, 1);
    double lower = neighbor_value(L, in, bc, i, j, k, AY, 0);
    double upper = neighbor_value(L, in, bc, i, j, k, AY, 1);
    double back = neighbor_value(L, in, bc, i, j, k, AZ, 0);
    double front = neighbor_value(L, in, bc, i, j, k, AZ, 1);
    out[IDX(L, i, j, k)] = -(right - 2.0 * center + left) / (dx * dx) -
                           (upper - 2.0 * center + lower) / (dy * dy) -
                           (front - 2.0 * center + back) / (dz * dz);
  }
}

/* compute_operator_diagonal (linsolve/poisson_solver.cpp:271-314) */
static void operator_diagonal(const lay_t* L, const oo_pbc* bc, double* diag) {
  FOR_ACTIVE(L) {
    double value = 0.0;
    for(int axis = 0; axis < 3; ++axis) {
      double inv = 1.0 / pow(L->h[axis], 2.0);
      double coefficient = 2.0 * inv;
      int c = axis == AX ? i : axis == AY ? j : k;
      int begin = 1, end = 1 + L->n[axis];
      if(bc->faces[2 * axis].type == OO_P_PERIODIC) {
        value += coefficient;
        continue;
      }
      if(c == begin)
        coefficient += bc->faces[2 * axis].type == OO_P_DIRICHLET ? inv : -inv;
      if(c == end - 1)
        coefficient += bc->faces[2 * axis + 1].type == OO_P_DIRICHLET ? inv : -inv;
      value += coefficient;
    }
    diag[IDX(L, i, j, k)] = value;
  }
}

/* HierarchyLevel (linsolve/poisson_solver.cpp:347-362) */
typedef struct {
  oo_grid grid;
  lay_t L;
  double *correction, *rhs, *residual, *scratch, *diagonal;
} level_t;

static int can_coarsen_axis(int cells) { return cells > 1 && cells % 2 == 0 && cells > 2; }

/* build_hierarchy / coarsen_grid / can_coarsen (linsolve/poisson_solver.cpp:316-384) */
static int build_hierarchy(const oo_grid* fine, const oo_pbc* hom, level_t* levels, int cap) {
  int count = 0;
  oo_grid g = *fine;
  for(;;) {
    level_t* lv = &levels[count++];
    lv->grid = g;
    lv->L = layout_of(&g, LOC_CELL);
    lv->correction = alloc_field(&lv->L);
    lv->rhs = alloc_field(&lv->L);
    lv->residual = alloc_field(&lv->L);
    lv->scratch = alloc_field(&lv->L);
    lv->diagonal = alloc_field(&lv->L);
    operator_diagonal(&lv->L, hom, lv->diagonal);
    if(count >= cap) break;
    if(!(can_coarsen_axis(g.nx) || can_coarsen_axis(g.ny) || can_coarsen_axis(g.nz))) break;
    oo_grid c = g;
    if(can_coarsen_axis(g.nx)) { c.nx = g.nx / 2; c.dx = 2.0 * g.dx; }
    if(can_coarsen_axis(g.ny)) { c.ny = g.ny / 2; c.dy = 2.0 * g.dy; }
    if(can_coarsen_axis(g.nz)) { c.nz = g.nz / 2; c.dz = 2.0 * g.dz; }
    if(c.nx == g.nx && c.ny == g.ny && c.nz == g.nz) break;
    g = c;
  }
  return count;
}

static void free_hierarchy(level_t* levels, int count) {
  for(int l = 0; l < count; ++l) {
    free(levels[l].correction);
    free(levels[l].rhs);
    free(levels[l].residual);
    free(levels[l].scratch);
    free(levels[l].diagonal);
  }
}

/* restrict_full_weighting (linsolve/poisson_solver.cpp:397-424) */
static void restrict_fw(const lay_t* F, const double* fine, const lay_t* C, double* coarse) {
  int rx = F->n[0] == C->n[0] ? 1 : 2, ry = F->n[1] == C->n[1] ? 1 : 2;
  int rz = F->n[2] == C->n[2] ? 1 : 2;
  double inv = 1.0 / (double)(rx * ry * rz);
  for(int kc = 0; kc < C->n[2]; ++kc)
    for(int jc = 0; jc < C->n[1]; ++jc)
      for(int ic = 0; ic < C->n[0]; ++ic) {
        double sum = 0.0;
        for(int dz = 0; dz < rz; ++dz)
          for(int dy = 0; dy < ry; ++dy)
            for(int dx = 0; dx < rx; ++dx)
              sum += fine[IDX(F, ic * rx + dx + 1, jc * ry + dy + 1, kc * rz + dz + 1)];
        coarse[IDX(C, ic + 1, jc + 1, kc + 1)] = inv * sum;
      }
}

/* prolongate_and_add (linsolve/poisson_solver.cpp:426-451) */
static void prolong_add(const lay_t* C, const double* coarse, const lay_t* F, double* fine) {
  int rx = F->n[0] == C->n[0] ? 1 : 2, ry = F->n[1] == C->n[1] ? 1 : 2;
  int rz = F->n[2] == C->n[2] ? 1 : 2;
  for(int kc = 0; kc < C->n[2]; ++kc)
    for(int jc = 0; jc < C->n[1]; ++jc)
      for(int ic = 0; ic < C->n[0]; ++ic) {
        double cv = coarse[IDX(C, ic + 1, jc + 1, kc + 1)];
        for(int dz = 0; dz < rz; ++dz)
          for(int dy = 0; dy < ry; ++dy)
            for(int dx = 0; dx < rx; ++dx)
              fine[IDX(F, ic * rx + dx + 1, jc * ry + dy + 1, kc * rz + dz + 1)] += cv;
      }
}

/* gaussian_elimination (linsolve/poisson_solver.cpp:482-528) */
static int gaussian_elimination(int n, double* m, double* rhs) {
  for(int pivot = 0; pivot < n; ++pivot) {
    int best = pivot;
    double best_abs = fabs(m[(size_t)pivot * n + pivot]);
    for(int row = pivot + 1; row < n; ++row) {
      double cand = fabs(m[(size_t)row * n + pivot]);
      if(cand > best_abs) {
        best = row;
        best_abs = cand;
      }
    }
    if(best_abs < kSmallNumber)
      return fail(ERUNTIME, "direct coarse solve encountered a singular matrix");
    if(best != pivot) {
      for(int c = 0; c < n; ++c) {
        double t = m[(size_t)pivot * n + c];
        m[(size_t)pivot * n + c] = m[(size_t)best * n + c];
        m[(size_t)best * n + c] = t;
      }
      double t = rhs[pivot];
      rhs[pivot] = rhs[best];
      rhs[best] = t;
    }
    double inv = 1.0 / m[(size_t)pivot * n + pivot];
    for(int row = pivot + 1; row < n; ++row) {
      double factor = m[(size_t)row * n + pivot] * inv;
      if(fabs(factor) < kSmallNumber) continue;
      for(int c = pivot; c < n; ++c) m[(size_t)row * n + c] -= factor * m[(size_t)pivot * n + c];
      rhs[row] -= factor * rhs[pivot];
    }
  }
  for(int row = n; row-- > 0;) {
    double sum = rhs[row];
    for(int c = row + 1; c < n; ++c) sum -= m[(size_t)row * n + c] * rhs[c];
    rhs[row] = sum / m[(size_t)row * n + row];
  }
  return OK;
}

/* direct_coarse_solve (linsolve/poisson_solver.cpp:530-567) */
static int direct_coarse_solve(level_t* lv, const oo_pbc* bc, int zero_mean) {
  const lay_t* L = &lv->L;
  int n = L->n[0] * L->n[1] * L->n[2];
  double* m = (double*)calloc((size_t)n * n, sizeof(double));
  double* sol = (double*)malloc((size_t)n * sizeof(double));
  double* basis = alloc_field(L);
  double* image = alloc_field(L);
  int q = 0;
  FOR_ACTIVE(L) sol[q++] = lv->rhs[IDX(L, i, j, k)];
  for(int col = 0; col < n; ++col) {
    fill_storage(L, basis, 0.0);
    q = 0;
    FOR_ACTIVE(L) basis[IDX(L, i, j, k)] = q++ == col ? 1.0 : 0.0;
    poisson_operator(L, basis, bc, image);
    q = 0;
    FOR_ACTIVE(L) m[(size_t)(q++) * n + col] = image[IDX(L, i, j, k)];
  }
  if(zero_mean) {
    for(int c = 0; c < n; ++c) m[(size_t)(n - 1) * n + c] = 1.0;
    sol[n - 1] = 0.0;
  }
  int rc = gaussian_elimination(n, m, sol);
  if(!rc) {
    fill_storage(L, lv->correction, 0.0);
    q = 0;
    FOR_ACTIVE(L) lv->correction[IDX(L, i, j, k)] = sol[q++];
    if(zero_mean) subtract_active_mean(L, lv->correction);
  }
  free(m);
  free(sol);
  free(basis);
  free(image);
  return rc;
}

static const double kJacobiOmega = 2.0 / 3.0;
enum { kPreSmoothing = 2, kPostSmoothing = 2 };

/* smooth_jacobi (linsolve/poisson_solver.cpp:569-595) */
static void smooth_jacobi(level_t* lv, const oo_pbc* bc, int iterations, int zero_mean) {
  const lay_t* L = &lv->L;
  for(int it = 0; it < iterations; ++it) {
    poisson_operator(L, lv->correction, bc, lv->scratch);
    copy_field(L, lv->residual, lv->rhs);
    axpy_active(L, lv->residual, lv->scratch, -1.0);
    FOR_ACTIVE(L) {
      size_t q = IDX(L, i, j, k);
      lv->scratch[q] = lv->correction[q] + kJacobiOmega * lv->residual[q] / lv->diagonal[q];
    }
    copy_active(L, lv->correction, lv->scratch);
    if(zero_mean) subtract_active_mean(L, lv->correction);
  }
}

/* v_cycle (linsolve/poisson_solver.cpp:597-633) */
static int v_cycle(level_t* levels, int count, int l, const oo_pbc* bc, int zero_mean) {
  level_t* lv = &levels[l];
  fill_storage(&lv->L, lv->correction, 0.0);
  if(l + 1 == count) return direct_coarse_solve(lv, bc, zero_mean);
  smooth_jacobi(lv, bc, kPreSmoothing, zero_mean);
  poisson_operator(&lv->L, lv->correction, bc, lv->scratch);
  copy_field(&lv->L, lv->residual, lv->rhs);
  axpy_active(&lv->L, lv->residual, lv->scratch, -1.0);
  if(zero_mean) subtract_active_mean(&lv->L, lv->residual);
  level_t* co = &levels[l + 1];
  fill_storage(&co->L, co->rhs, 0.0);
  fill_storage(&co->L, co->correction, 0.0);
  restrict_fw(&lv->L, lv->residual, &co->L, co->rhs);
  if(zero_mean) subtract_active_mean(&co->L, co->rhs);
  int rc = v_cycle(levels, count, l + 1, bc, zero_mean);
  if(rc) return rc;
  prolong_add(&co->L, co->correction, &lv->L, lv->correction);
  if(zero_mean) subtract_active_mean(&lv->L, lv->correction);
  smooth_jacobi(lv, bc, kPostSmoothing, zero_mean);
  return OK;
}

/* solve_pressure_poisson (linsolve/poisson_solver.cpp:678-809) */
static int poisson_solve(const oo_grid* g, const oo_pbc* pbc, int max_it, double tol,
                         const double* rhs, double* pressure, oo_poisson_diag* d, double* hist,
                         int hist_cap) {
  if(max_it <= 0) return fail(EINVAL_, "solve_pressure_poisson expects iterations > 0");
  if(tol <= 0.0) return fail(EINVAL_, "solve_pressure_poisson expects tolerance > 0");
  for(int axis = 0; axis < 3; ++axis) {
    int periodic = 0;
    int rc = pressure_axis_periodic(pbc, axis, &periodic);
    if(rc) return rc;
  }
  memset(d, 0, sizeof(*d));
  lay_t L = layout_of(g, LOC_CELL);
  oo_pbc hom = *pbc;
  for(int f = 0; f < 6; ++f) {
    hom.faces[f].value = 0.0;
    hom.faces[f].gradient = 0.0;
  }
  int zero_mean = 1;
  for(int f = 0; f < 6; ++f)
    if(pbc->faces[f].type == OO_P_DIRICHLET) zero_mean = 0;

  double* system_rhs = alloc_field(&L);
  double* residual = alloc_field(&L);
  double* search = alloc_field(&L);
  double* opres = alloc_field(&L);
  double* precond = alloc_field(&L);
  double* zero = alloc_field(&L);
  double* source = alloc_field(&L);
  poisson_operator(&L, zero, pbc, source); /* build_boundary_source (:635-642) */

  copy_active(&L, system_rhs, rhs);
  scale_active(&L, system_rhs, -1.0);
  axpy_active(&L, system_rhs, source, -1.0);

  d->zero_mean_enforced = zero_mean;
  d->pre_smoothing_steps = kPreSmoothing;
  d->post_smoothing_steps = kPostSmoothing;

  level_t levels[64];
  int count = build_hierarchy(g, &hom, levels, 64);
  d->multigrid_levels = count;
  d->coarse_unknowns = levels[count - 1].grid.nx * levels[count - 1].grid.ny * levels[count - 1].grid.nz;

  if(zero_mean) {
    d->removed_rhs_mean = subtract_active_mean(&L, system_rhs);
    subtract_active_mean(&L, pressure);
  }
  poisson_operator(&L, pressure, &hom, opres);
  copy_field(&L, residual, system_rhs);
  axpy_active(&L, residual, opres, -1.0);
  if(zero_mean) subtract_active_mean(&L, residual);

  d->initial_residual_l2 = active_l2_norm(&L, residual);
  d->final_residual_l2 = d->initial_residual_l2;
  d->relative_residual = d->initial_residual_l2 > 0.0 ? 1.0 : 0.0;
  int nhist = 0;
  if(hist && nhist < hist_cap) hist[nhist] = d->initial_residual_l2;
  ++nhist;

  int rc = OK;
  if(d->initial_residual_l2 <= tol) {
    d->converged = 1;
    d->relative_residual = 0.0;
    goto done;
  }

  copy_field(&L, levels[0].rhs, residual);
  rc = v_cycle(levels, count, 0, &hom, zero_mean);
  if(rc) goto done;
  copy_field(&L, precond, levels[0].correction);
  if(zero_mean) subtract_active_mean(&L, precond);
  copy_field(&L, search, precond);

  double rz = dot_active(&L, residual, precond);
  for(int it = 0; it < max_it; ++it) {
    poisson_operator(&L, search, &hom, opres);
    if(zero_mean) subtract_active_mean(&L, opres);
    double search_dot = dot_active(&L, search, opres);
    if(fabs(search_dot) < kSmallNumber) break;
    double alpha = rz / search_dot;
    axpy_active(&L, pressure, search, alpha);
    if(zero_mean) subtract_active_mean(&L, pressure);
    axpy_active(&L, residual, opres, -alpha);
    if(zero_mean) subtract_active_mean(&L, residual);
    d->iterations = it + 1;
    d->final_residual_l2 = active_l2_norm(&L, residual);
    d->relative_residual = d->initial_residual_l2 > 0.0
                               ? d->final_residual_l2 / d->initial_residual_l2
                               : 0.0;
    if(hist && nhist < hist_cap) hist[nhist] = d->final_residual_l2;
    ++nhist;
    if(d->relative_residual <= tol) {
      d->converged = 1;
      break;
    }
    copy_field(&L, levels[0].rhs, residual);
    rc = v_cycle(levels, count, 0, &hom, zero_mean);
    if(rc) goto done;
    copy_field(&L, precond, levels[0].correction);
    if(zero_mean) subtract_active_mean(&L, precond);
    double next = dot_active(&L, residual, precond);
    double beta = next / rz;
    FOR_ACTIVE(&L) {
      size_t q = IDX(&L, i, j, k);
      search[q] = precond[q] + beta * search[q];
    }
    if(zero_mean) subtract_active_mean(&L, search);
    rz = next;
  }

done:
  free_hierarchy(levels, count);
  free(system_rhs);
  free(residual);
  free(search);
  free(opres);
  free(precond);
  free(zero);
  free(source);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* projection (solver/projection.cpp:1049-1131)                              */
/* ------------------------------------------------------------------------ */

/* build_pressure_rhs (solver/projection.cpp:1049-1064) */
static int build_pressure_rhs(const oo_grid* g, const oo_bc* bc, double dt, double density,
                              const double* u, const double* v, const double* w, double* rhs) {
  if(dt <= 0.0) return fail(EINVAL_, "build_pressure_rhs expects dt > 0");
  if(density <= 0.0) return fail(EINVAL_, "build_pressure_rhs expects density > 0");
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  lay_t P = layout_of(g, LOC_CELL);
  double* wu = clone_field(&U, u);
  double* wv = clone_field(&V, v);
  double* ww = clone_field(&W, w);
  int rc = velocity_bc(g, bc, wu, wv, ww);
  if(!rc) {
    divergence(g, wu, wv, ww, rhs);
    scale_active(&P, rhs, density / dt);
  }
  free(wu);
  free(wv);
  free(ww);
  return rc;
}

/* correct_velocity (solver/projection.cpp:1066-1095) */
static int correct_velocity(const oo_grid* g, const oo_bc* bc, double dt, double density,
                            const double* pu, const double* pv, const double* pw,
                            const double* phi, double* cu, double* cv, double* cw) {
  if(dt <= 0.0) return fail(EINVAL_, "correct_velocity expects dt > 0");
  if(density <= 0.0) return fail(EINVAL_, "correct_velocity expects density > 0");
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  lay_t P = layout_of(g, LOC_CELL);
  oo_pbc pbc;
  int rc = derive_pbc(bc, &pbc);
  if(rc) return rc;
  double* pg = clone_field(&P, phi);
  rc = pressure_bc(g, &pbc, pg);
  if(rc) {
    free(pg);
    return rc;
  }
  double* gu = alloc_field(&U);
  double* gv = alloc_field(&V);
  double* gw = alloc_field(&W);
  gradient(g, pg, gu, gv, gw);
  copy_field(&U, cu, pu);
  copy_field(&V, cv, pv);
  copy_field(&W, cw, pw);
  double scale = -dt / density;
  axpy_active(&U, cu, gu, scale);
  axpy_active(&V, cv, gv, scale);
  axpy_active(&W, cw, gw, scale);
  rc = velocity_bc(g, bc, cu, cv, cw);
  free(pg);
  free(gu);
  free(gv);
  free(gw);
  return rc;
}

static int project_velocity(const oo_grid* g, const oo_bc* bc, double dt, double density,
                            int max_it, double tol, const double* pu, const double* pv,
                            const double* pw, double* phi, double* cu, double* cv, double* cw,
                            double* rhs_out, oo_projection_diag* d) {
  lay_t U = layout_of(g, LOC_FX), V = layout_of(g, LOC_FY), W = layout_of(g, LOC_FZ);
  lay_t P = layout_of(g, LOC_CELL);
  memset(d, 0, sizeof(*d));
  oo_pbc pbc;
  int rc = derive_pbc(bc, &pbc);
  if(rc) return rc;
  double* rhs = alloc_field(&P);
  double* div = alloc_field(&P);
  double* wu = clone_field(&U, pu);
  double* wv = clone_field(&V, pv);
  double* ww = clone_field(&W, pw);
  rc = velocity_bc(g, bc, wu, wv, ww);
  if(rc) goto done;
  divergence(g, wu, wv, ww, div);
  d->divergence_l2_before = active_l2_norm(&P, div);
  rc = build_pressure_rhs(g, bc, dt, density, wu, wv, ww, rhs);
  if(rc) goto done;
  d->rhs_l2 = active_l2_norm(&P, rhs);
  rc = poisson_solve(g, &pbc, max_it, tol, rhs, phi, &d->pressure_solve, NULL, 0);
  if(rc) goto done;
  rc = correct_velocity(g, bc, dt, density, wu, wv, ww, phi, cu, cv, cw);
  if(rc) goto done;
  divergence(g, cu, cv, cw, div);
  d->divergence_l2_after = active_l2_norm(&P, div);
  d->pressure_mean = active_mean(&P, phi);
  if(rhs_out) copy_active(&P, rhs_out, rhs);
done:
  free(rhs);
  free(div);
  free(wu);
  free(wv);
  free(ww);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* step drivers                                                             */
/* ------------------------------------------------------------------------ */

static double max_velocity_change(const oo_grid* g, const double* a[3], const double* b[3]) {
  double change = 0.0;
  for(int c = 0; c < 3; ++c) {
    lay_t L = layout_of(g, LOC_FX + c);
    FOR_ACTIVE(&L) {
      double d = fabs(a[c][IDX(&L, i, j, k)] - b[c][IDX(&L, i, j, k)]);
      if(d > change) change = d;
    }
  }
  return change;
}

/* second_derivative_axis / mixed / triple (solver/taylor_green.cpp:132-194) */
static double d2_axis(const lay_t* L, const double* f, int i, int j, int k, int axis) {
  double spacing = L->h[axis];
  double inv = 1.0 / (spacing * spacing);
  int di = axis == AX, dj = axis == AY, dk = axis == AZ;
  return (f[IDX(L, i + di, j + dj, k + dk)] - 2.0 * f[IDX(L, i, j, k)] +
          f[IDX(L, i - di, j - dj, k - dk)]) *
         inv;
}

static double d2_mixed(const lay_t* L, const double* f, int i, int j, int k, int outer, int inner) {
  double spacing = L->h[outer];
  double inv = 1.0 / (spacing * spacing);
  int di = outer == AX, dj = outer == AY, dk = outer == AZ;
  return (d2_axis(L, f, i + di, j + dj, k + dk, inner) - 2.0 * d2_axis(L, f, i, j, k, inner) +
          d2_axis(L, f, i - di, j - dj, k - dk, inner)) *
         inv;
}

static double d2_triple(const lay_t* L, const double* f, int i, int j, int k, int a, int b, int c) {
  double spacing = L->h[a];
  double inv = 1.0 / (spacing * spacing);
  int di = a == AX, dj = a == AY, dk = a == AZ;
  return (d2_mixed(L, f, i + di, j + dj, k + dk, b, c) - 2.0 * d2_mixed(L, f, i, j, k, b, c) +
          d2_mixed(L, f, i - di, j - dj, k - dk, b, c)) *
         inv;
}

/* mixed_second_derivative_2d (solver/lid_driven_cavity.cpp:219-232): the
 * cavity variant divides by dy^2 instead of multiplying by its inverse. */
static double d2_mixed_cavity(const lay_t* L, const double* f, int i, int j, int k) {
  double dy = L->h[1];
  double dy2 = dy * dy;
  double im1 = (f[IDX(L, i - 1, j + 1, k)] - 2.0 * f[IDX(L, i - 1, j, k)] + f[IDX(L, i - 1, j - 1, k)]) / dy2;
  double i0 = (f[IDX(L, i, j + 1, k)] - 2.0 * f[IDX(L, i, j, k)] + f[IDX(L, i, j - 1, k)]) / dy2;
  double ip1 = (f[IDX(L, i + 1, j + 1, k)] - 2.0 * f[IDX(L, i + 1, j, k)] + f[IDX(L, i + 1, j - 1, k)]) / dy2;
  double dx = L->h[0];
  double inv = 1.0 / (dx * dx);
  return (ip1 - 2.0 * i0 + im1) * inv;
}

enum { CORR_TG = 0, CORR_CAVITY = 1 };

/* compute_factorized_correction (solver/taylor_green.cpp:196-225) and
 * compute_factorized_correction_2d (solver/lid_driven_cavity.cpp:234-252) */
static void factorized_correction(const oo_grid* g, int variant, double alpha, const double* in[3],
                                  double* out[3]) {
  int three_d = g->nz != 1;
  for(int c = 0; c < 3; ++c) {
    lay_t L = layout_of(g, LOC_FX + c);
    fill_storage(&L, out[c], 0.0);
    FOR_ACTIVE(&L) {
      double corr;
      if(variant == CORR_CAVITY) {
        corr = d2_mixed_cavity(&L, in[c], i, j, k);
      } else {
        corr = d2_mixed(&L, in[c], i, j, k, AX, AY);
        if(three_d) {
          corr += d2_mixed(&L, in[c], i, j, k, AX, AZ);
          corr += d2_mixed(&L, in[c], i, j, k, AY, AZ);
          corr -= alpha * d2_triple(&L, in[c], i, j, k, AX, AY, AZ);
        }
      }
      out[c][IDX(&L, i, j, k)] = corr;
    }
  }
}

typedef struct {
  oo_grid g;
  oo_bc bc;
  double viscosity, dt;
  int max_it;
  double tol;
  int variant;
  const char* name;
} driver_t;

/* One step of run_taylor_green_steps (solver/taylor_green.cpp:577-633) or of
 * advance_lid_driven_cavity_impl (solver/lid_driven_cavity.cpp:562-623). */
static int run_steps(const driver_t* D, int steps, oo_state* s, int track_max_div) {
  const oo_grid* g = &D->g;
  lay_t Lc[3] = {layout_of(g, LOC_FX), layout_of(g, LOC_FY), layout_of(g, LOC_FZ)};
  lay_t P = layout_of(g, LOC_CELL);
  double* vel[3] = {s->u, s->v, s->w};
  double* prev[3] = {s->adv_u, s->adv_v, s->adv_w};
  double *cur[3], *adv[3], *dif[3], *grad[3], *corr[3], *rhs[3], *pred[3], *corrected[3];
  for(int c = 0; c < 3; ++c) {
    cur[c] = alloc_field(&Lc[c]);
    adv[c] = alloc_field(&Lc[c]);
    dif[c] = alloc_field(&Lc[c]);
    grad[c] = alloc_field(&Lc[c]);
    corr[c] = alloc_field(&Lc[c]);
    rhs[c] = alloc_field(&Lc[c]);
    pred[c] = alloc_field(&Lc[c]);
    corrected[c] = alloc_field(&Lc[c]);
  }
  double* pc = alloc_field(&P);
  double* prhs = alloc_field(&P);
  double dt = D->dt;
  double alpha = 0.5 * D->viscosity * dt;
  int rc = OK;
  for(int step = 0; step < steps && !rc; ++step) {
    for(int c = 0; c < 3; ++c) copy_field(&Lc[c], cur[c], vel[c]);
    rc = velocity_bc(g, &D->bc, cur[0], cur[1], cur[2]);
    if(rc) break;
    /* assemble_predictor_rhs (solver/taylor_green.cpp:227-256) */
    advection(g, cur[0], cur[1], cur[2], adv[0], adv[1], adv[2]);
    diffusion(g, D->viscosity, cur[0], cur[1], cur[2], dif[0], dif[1], dif[2]);
    gradient(g, s->p, grad[0], grad[1], grad[2]);
    factorized_correction(g, D->variant, alpha, (const double**)cur, corr);
    for(int c = 0; c < 3; ++c) {
      copy_field(&Lc[c], rhs[c], cur[c]);
    }
    for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], grad[c], -dt);
    for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], dif[c], 0.5 * dt);
    if(s->has_previous_advection) {
      for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], adv[c], -1.5 * dt);
      for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], prev[c], 0.5 * dt);
    } else {
      for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], adv[c], -dt);
    }
    for(int c = 0; c < 3; ++c) axpy_active(&Lc[c], rhs[c], corr[c], alpha * alpha);

    int line_solves = 0;
    rc = predictor_adi(g, &D->bc, alpha, rhs[0], rhs[1], rhs[2], pred[0], pred[1], pred[2],
                       &line_solves);
    if(rc) break;
    fill_storage(&P, pc, 0.0);
    oo_projection_diag pd;
    rc = project_velocity(g, &D->bc, dt, 1.0, D->max_it, D->tol, pred[0], pred[1], pred[2], pc,
                          corrected[0], corrected[1], corrected[2], prhs, &pd);
    if(rc) break;
    /* require_converged_pressure_projection (solver/projection.cpp:1133-1147) */
    if(!pd.pressure_solve.converged) {
      rc = fail(ERUNTIME,
                "%s pressure solve did not converge at step %d (iterations=%d, "
                "relative_residual=%g, tolerance=%g)",
                D->name, step + 1, pd.pressure_solve.iterations,
                pd.pressure_solve.relative_residual, D->tol);
      break;
    }
    axpy_active(&P, s->p, pc, 1.0);
    axpy_active(&P, s->p, prhs, -0.5 * D->viscosity * dt);
    diffusion(g, D->viscosity, corrected[0], corrected[1], corrected[2], dif[0], dif[1], dif[2]);
    rc = total_pressure_bc(g, &D->bc, dif[0], dif[1], dif[2], s->p);
    if(rc) break;
    double cfl = advective_cfl(g, corrected[0], corrected[1], corrected[2], dt);
    double delta =
        max_velocity_change(g, (const double**)vel, (const double**)corrected);
    if(!isfinite(delta) || !isfinite(pd.divergence_l2_after)) {
      rc = fail(ERUNTIME, "%s solve produced a non-finite state", D->name);
      break;
    }
    for(int c = 0; c < 3; ++c) {
      copy_field(&Lc[c], vel[c], corrected[c]);
      copy_field(&Lc[c], prev[c], adv[c]);
    }
    s->has_previous_advection = 1;
    oo_step_metrics* m = &s->metrics;
    m->step += 1;
    m->time += dt;
    m->dt = dt;
    m->max_cfl = cfl;
    m->max_velocity_change = delta;
    m->divergence_l2 = pd.divergence_l2_after;
    if(track_max_div)
      m->max_divergence_l2 = m->max_divergence_l2 < pd.divergence_l2_after
                                 ? pd.divergence_l2_after
                                 : m->max_divergence_l2;
    m->pressure_iterations = pd.pressure_solve.iterations;
    m->pressure_relative_residual = pd.pressure_solve.relative_residual;
  }
  for(int c = 0; c < 3; ++c) {
    free(cur[c]);
    free(adv[c]);
    free(dif[c]);
    free(grad[c]);
    free(corr[c]);
    free(rhs[c]);
    free(pred[c]);
    free(corrected[c]);
  }
  free(pc);
  free(prhs);
  return rc;
}

/* ---- Taylor-Green (solver/taylor_green.cpp) ---- */

static double pi_(void) { return acos(-1.0); }

static int tg_validate(const oo_tg_config* c) {
  if(c->nx <= 0 || c->ny <= 0 || c->nz <= 0)
    return fail(EINVAL_, "Taylor-Green config expects positive nx, ny, and nz");
  if(c->viscosity <= 0.0) return fail(EINVAL_, "Taylor-Green config expects viscosity > 0");
  if(c->cfl_limit <= 0.0) return fail(EINVAL_, "Taylor-Green config expects cfl_limit > 0");
  if(c->final_time <= 0.0) return fail(EINVAL_, "Taylor-Green config expects final_time > 0");
  if(c->poisson_max_iterations <= 0 || c->poisson_tolerance <= 0.0)
    return fail(EINVAL_, "Taylor-Green config expects positive Poisson controls");
  return OK;
}

/* make_taylor_green_grid (solver/taylor_green.cpp:497-508) */
int oo_tg_grid(const oo_tg_config* c, oo_grid* g) {
  int rc = tg_validate(c);
  if(rc) return rc;
  double len = 2.0 * pi_();
  g->nx = c->nx;
  g->ny = c->ny;
  g->nz = c->nz;
  g->dx = len / (double)c->nx;
  g->dy = len / (double)c->ny;
  g->dz = c->nz > 1 ? len / (double)c->nz : 1.0;
  return OK;
}

/* taylor_green_dt (solver/taylor_green.cpp:397-401, 519-525) */
double oo_tg_dt(const oo_tg_config* c) {
  oo_grid g;
  if(oo_tg_grid(c, &g)) return 0.0;
  double inverse_sum = 1.0 / g.dx + 1.0 / g.dy + (g.nz == 1 ? 0.0 : 1.0 / g.dz);
  double dt_upper = c->cfl_limit / inverse_sum;
  int steps = (int)ceil(c->final_time / dt_upper);
  if(steps < 1) steps = 1;
  return c->final_time / (double)steps;
}

/* make_taylor_green_boundary_conditions (solver/taylor_green.cpp:510-517) */
int oo_tg_bc(const oo_tg_config* c, oo_bc* bc) {
  memset(bc, 0, sizeof(*bc));
  for(int f = 0; f < 6; ++f) bc->faces[f].type = OO_PERIODIC;
  if(c->nz <= 1) {
    bc->faces[4].type = OO_SYMMETRY;
    bc->faces[5].type = OO_SYMMETRY;
  }
  return OK;
}

static double coord(const lay_t* L, int axis, int storage_index) {
  int shifted = storage_index - 1;
  int normal = L->loc == LOC_FX ? AX : L->loc == LOC_FY ? AY : L->loc == LOC_FZ ? AZ : -1;
  if(axis == normal) return (double)shifted * L->h[axis];
  return ((double)shifted + 0.5) * L->h[axis];
}

int oo_tg_init_tail(const oo_tg_config* c, oo_state* s) {
  oo_grid g;
  int rc = oo_tg_grid(c, &g);
  if(rc) return rc;
  oo_bc bc;
  oo_tg_bc(c, &bc);
  rc = velocity_bc(&g, &bc, s->u, s->v, s->w);
  if(rc) return rc;
  lay_t U = layout_of(&g, LOC_FX), V = layout_of(&g, LOC_FY), W = layout_of(&g, LOC_FZ);
  double* du = alloc_field(&U);
  double* dv = alloc_field(&V);
  double* dw = alloc_field(&W);
  diffusion(&g, c->viscosity, s->u, s->v, s->w, du, dv, dw);
  rc = total_pressure_bc(&g, &bc, du, dv, dw, s->p);
  free(du);
  free(dv);
  free(dw);
  return rc;
}

/* initialize_exact_state (solver/taylor_green.cpp:335-395) */
int oo_tg_init(const oo_tg_config* c, int mode, oo_state* s) {
  oo_grid g;
  int rc = oo_tg_grid(c, &g);
  if(rc) return rc;
  lay_t U = layout_of(&g, LOC_FX), V = layout_of(&g, LOC_FY), W = layout_of(&g, LOC_FZ);
  lay_t P = layout_of(&g, LOC_CELL);
  int three_d = c->nz > 1;
  double decay = exp(-(three_d ? 3.0 : 2.0) * c->viscosity * 0.0);
  fill_storage(&U, s->u, 0.0);
  fill_storage(&V, s->v, 0.0);
  fill_storage(&W, s->w, 0.0);
  fill_storage(&P, s->p, 0.0);
  fill_storage(&U, s->adv_u, 0.0);
  fill_storage(&V, s->adv_v, 0.0);
  fill_storage(&W, s->adv_w, 0.0);
  FOR_ACTIVE(&U) {
    double z = coord(&U, AZ, k), y = coord(&U, AY, j), x = coord(&U, AX, i);
    double zf = three_d ? cos(z) : 1.0;
    s->u[IDX(&U, i, j, k)] = mode == 0 ? -cos(x) * sin(y) * zf * decay : sin(x) * cos(y) * zf * decay;
  }
  FOR_ACTIVE(&V) {
    double z = coord(&V, AZ, k), y = coord(&V, AY, j), x = coord(&V, AX, i);
    double zf = three_d ? cos(z) : 1.0;
    s->v[IDX(&V, i, j, k)] = mode == 0 ? sin(x) * cos(y) * zf * decay : -cos(x) * sin(y) * zf * decay;
  }
  double pdecay = exp((three_d ? -6.0 : -4.0) * c->viscosity * 0.0);
  double sign = mode == 0 ? 1.0 : -1.0;
  FOR_ACTIVE(&P) {
    double z = coord(&P, AZ, k), y = coord(&P, AY, j), x = coord(&P, AX, i);
    if(three_d)
      s->p[IDX(&P, i, j, k)] =
          sign * -0.0625 * (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0) * pdecay;
    else
      s->p[IDX(&P, i, j, k)] = sign * -0.25 * (cos(2.0 * x) + cos(2.0 * y)) * pdecay;
  }
  s->has_previous_advection = 0;
  memset(&s->metrics, 0, sizeof(s->metrics));
  s->metrics.dt = oo_tg_dt(c);
  return oo_tg_init_tail(c, s);
}

int oo_tg_steps(const oo_tg_config* c, int steps, oo_state* s) {
  int rc = tg_validate(c);
  if(rc) return rc;
  if(steps < 0) return fail(EINVAL_, "run_taylor_green_steps expects a non-negative step count");
  driver_t D;
  oo_tg_grid(c, &D.g);
  oo_tg_bc(c, &D.bc);
  D.viscosity = c->viscosity;
  D.dt = oo_tg_dt(c);
  D.max_it = c->poisson_max_iterations;
  D.tol = c->poisson_tolerance;
  D.variant = CORR_TG;
  D.name = "Taylor-Green";
  return run_steps(&D, steps, s, 1);
}

/* kinetic_energy / exact_* / velocity_relative_l2_error / build_validation
 * (solver/taylor_green.cpp:258-333, 403-417) */
int oo_tg_validate(const oo_tg_config* c, int mode, const double* u, const double* v,
                   const double* w, double time, oo_tg_validation* out) {
  oo_grid g;
  int rc = oo_tg_grid(c, &g);
  if(rc) return rc;
  int three_d = c->nz > 1;
  lay_t P = layout_of(&g, LOC_CELL);
  lay_t U = layout_of(&g, LOC_FX), V = layout_of(&g, LOC_FY), W = layout_of(&g, LOC_FZ);
  double energy_sum = 0.0;
  size_t count = 0;
  FOR_ACTIVE(&P) {
    double uc = 0.5 * (u[IDX(&U, i, j, k)] + u[IDX(&U, i + 1, j, k)]);
    double vc = 0.5 * (v[IDX(&V, i, j, k)] + v[IDX(&V, i, j + 1, k)]);
    double wc = 0.5 * (w[IDX(&W, i, j, k)] + w[IDX(&W, i, j, k + 1)]);
    energy_sum += 0.5 * (uc * uc + vc * vc + wc * wc);
    ++count;
  }
  double ke = energy_sum / (double)count;
  double exact = (three_d ? 0.125 : 0.25) * exp(-(three_d ? 6.0 : 4.0) * c->viscosity * time);
  double decay = exp(-(three_d ? 3.0 : 2.0) * c->viscosity * time);
  double num = 0.0, den = 0.0;
  FOR_ACTIVE(&U) {
    double z = coord(&U, AZ, k), y = coord(&U, AY, j), x = coord(&U, AX, i);
    double ref;
    if(mode == 0) ref = three_d ? -cos(x) * sin(y) * cos(z) * decay : -cos(x) * sin(y) * decay;
    else ref = three_d ? sin(x) * cos(y) * cos(z) * decay : sin(x) * cos(y) * decay;
    double d = u[IDX(&U, i, j, k)] - ref;
    num += d * d;
    den += ref * ref;
  }
  FOR_ACTIVE(&V) {
    double z = coord(&V, AZ, k), y = coord(&V, AY, j), x = coord(&V, AX, i);
    double ref;
    if(mode == 0) ref = three_d ? sin(x) * cos(y) * cos(z) * decay : sin(x) * cos(y) * decay;
    else ref = three_d ? -cos(x) * sin(y) * cos(z) * decay : -cos(x) * sin(y) * decay;
    double d = v[IDX(&V, i, j, k)] - ref;
    num += d * d;
    den += ref * ref;
  }
  FOR_ACTIVE(&W) {
    double d = w[IDX(&W, i, j, k)];
    num += d * d;
  }
  out->kinetic_energy = ke;
  out->exact_kinetic_energy = exact;
  out->normalized_energy_error = fabs(ke - exact) / exact;
  out->velocity_relative_l2_error = den > 0.0 ? sqrt(num / den) : sqrt(num);
  return OK;
}

/* ---- lid-driven cavity (solver/lid_driven_cavity.cpp) ---- */

static int cavity_validate(const oo_cavity_config* c) {
  if(c->nx <= 0 || c->ny <= 0) return fail(EINVAL_, "lid-driven cavity config expects positive nx and ny");
  if(c->reynolds <= 0.0) return fail(EINVAL_, "lid-driven cavity config expects reynolds > 0");
  if(c->lid_velocity <= 0.0) return fail(EINVAL_, "lid-driven cavity config expects lid_velocity > 0");
  if(c->cfl_limit <= 0.0) return fail(EINVAL_, "lid-driven cavity config expects cfl_limit > 0");
  if(c->max_steps <= 0 || c->min_steps < 0)
    return fail(EINVAL_, "lid-driven cavity config expects non-negative step controls");
  if(c->poisson_max_iterations <= 0 || c->poisson_tolerance <= 0.0)
    return fail(EINVAL_, "lid-driven cavity config expects positive Poisson controls");
  return OK;
}

int oo_cavity_grid(const oo_cavity_config* c, oo_grid* g) {
  g->nx = c->nx;
  g->ny = c->ny;
  g->nz = 1;
  g->dx = 1.0 / (double)c->nx;
  g->dy = 1.0 / (double)c->ny;
  g->dz = 1.0;
  return OK;
}

double oo_cavity_dt(const oo_cavity_config* c) {
  oo_grid g;
  oo_cavity_grid(c, &g);
  double denominator = c->lid_velocity / g.dx + c->lid_velocity / g.dy;
  return c->cfl_limit / denominator;
}

/* make_lid_driven_cavity_boundary_conditions (solver/lid_driven_cavity.cpp:362-370) */
int oo_cavity_bc(const oo_cavity_config* c, oo_bc* bc) {
  memset(bc, 0, sizeof(*bc));
  for(int f = 0; f < 6; ++f) bc->faces[f].type = OO_NO_SLIP_WALL;
  bc->faces[3].type = OO_PRESCRIBED_VELOCITY;
  bc->faces[3].velocity[0] = c->lid_velocity;
  bc->faces[4].type = OO_SYMMETRY;
  bc->faces[5].type = OO_SYMMETRY;
  return OK;
}

/* initialize_lid_driven_cavity_state (solver/lid_driven_cavity.cpp:390-409) */
int oo_cavity_init(const oo_cavity_config* c, oo_state* s) {
  int rc = cavity_validate(c);
  if(rc) return rc;
  oo_grid g;
  oo_cavity_grid(c, &g);
  oo_bc bc;
  oo_cavity_bc(c, &bc);
  lay_t U = layout_of(&g, LOC_FX), V = layout_of(&g, LOC_FY), W = layout_of(&g, LOC_FZ);
  lay_t P = layout_of(&g, LOC_CELL);
  fill_storage(&U, s->u, 0.0);
  fill_storage(&V, s->v, 0.0);
  fill_storage(&W, s->w, 0.0);
  fill_storage(&U, s->adv_u, 0.0);
  fill_storage(&V, s->adv_v, 0.0);
  fill_storage(&W, s->adv_w, 0.0);
  fill_storage(&P, s->p, 0.0);
  s->has_previous_advection = 0;
  memset(&s->metrics, 0, sizeof(s->metrics));
  s->metrics.dt = oo_cavity_dt(c);
  rc = velocity_bc(&g, &bc, s->u, s->v, s->w);
  if(rc) return rc;
  double* du = alloc_field(&U);
  double* dv = alloc_field(&V);
  double* dw = alloc_field(&W);
  diffusion(&g, c->lid_velocity / c->reynolds, s->u, s->v, s->w, du, dv, dw);
  rc = total_pressure_bc(&g, &bc, du, dv, dw, s->p);
  free(du);
  free(dv);
  free(dw);
  return rc;
}

int oo_cavity_steps(const oo_cavity_config* c, int steps, oo_state* s) {
  int rc = cavity_validate(c);
  if(rc) return rc;
  if(steps < 0)
    return fail(EINVAL_, "run_lid_driven_cavity_steps expects a non-negative step count");
  driver_t D;
  oo_cavity_grid(c, &D.g);
  oo_cavity_bc(c, &D.bc);
  D.viscosity = c->lid_velocity / c->reynolds;
  D.dt = oo_cavity_dt(c);
  D.max_it = c->poisson_max_iterations;
  D.tol = c->poisson_tolerance;
  D.variant = CORR_CAVITY;
  D.name = "lid-driven cavity";
  return run_steps(&D, steps, s, 0);
}

/* ------------------------------------------------------------------------ */
/* exported operator entry points                                           */
/* ------------------------------------------------------------------------ */

int oo_advection(const oo_grid* g, const double* u, const double* v, const double* w,
                 double* au, double* av, double* aw) {
  int rc = check_grid(g);
  if(rc) return rc;
  advection(g, u, v, w, au, av, aw);
  return OK;
}

int oo_diffusion(const oo_grid* g, double nu, const double* u, const double* v, const double* w,
                 double* du, double* dv, double* dw) {
  int rc = check_grid(g);
  if(rc) return rc;
  diffusion(g, nu, u, v, w, du, dv, dw);
  return OK;
}

int oo_apply_velocity_bc(const oo_grid* g, const oo_bc* bc, double* u, double* v, double* w) {
  int rc = check_grid(g);
  if(rc) return rc;
  return velocity_bc(g, bc, u, v, w);
}

int oo_apply_pressure_bc(const oo_grid* g, const oo_pbc* pbc, double* p) {
  int rc = check_grid(g);
  if(rc) return rc;
  return pressure_bc(g, pbc, p);
}

int oo_derive_pressure_correction_bc(const oo_bc* bc, oo_pbc* out) { return derive_pbc(bc, out); }

int oo_apply_total_pressure_bc(const oo_grid* g, const oo_bc* bc, const double* su,
                               const double* sv, const double* sw, double* p) {
  int rc = check_grid(g);
  if(rc) return rc;
  return total_pressure_bc(g, bc, su, sv, sw, p);
}

int oo_gradient(const oo_grid* g, const double* p, double* gu, double* gv, double* gw) {
  int rc = check_grid(g);
  if(rc) return rc;
  gradient(g, p, gu, gv, gw);
  return OK;
}

int oo_divergence(const oo_grid* g, const double* u, const double* v, const double* w,
                  double* div) {
  int rc = check_grid(g);
  if(rc) return rc;
  divergence(g, u, v, w, div);
  return OK;
}

int oo_predictor_adi(const oo_grid* g, const oo_bc* bc, double alpha, const double* ru,
                     const double* rv, const double* rw, double* pu, double* pv, double* pw,
                     int* line_solves) {
  int rc = check_grid(g);
  if(rc) return rc;
  int ls = 0;
  rc = predictor_adi(g, bc, alpha, ru, rv, rw, pu, pv, pw, &ls);
  if(line_solves) *line_solves = ls;
  return rc;
}

int oo_poisson_solve(const oo_grid* g, const oo_pbc* pbc, int max_iterations, double tolerance,
                     const double* rhs, double* pressure, oo_poisson_diag* diag, double* hist,
                     int hist_cap) {
  int rc = check_grid(g);
  if(rc) return rc;
  oo_poisson_diag d;
  rc = poisson_solve(g, pbc, max_iterations, tolerance, rhs, pressure, &d, hist, hist_cap);
  if(diag) *diag = d;
  return rc;
}

int oo_project_velocity(const oo_grid* g, const oo_bc* bc, double dt, double density,
                        int max_iterations, double tolerance, const double* pu,
                        const double* pv, const double* pw, double* phi, double* cu,
                        double* cv, double* cw, double* rhs_out, oo_projection_diag* diag) {
  int rc = check_grid(g);
  if(rc) return rc;
  oo_projection_diag d;
  rc = project_velocity(g, bc, dt, density, max_iterations, tolerance, pu, pv, pw, phi, cu, cv, cw,
                        rhs_out, &d);
  if(diag) *diag = d;
  return rc;
}

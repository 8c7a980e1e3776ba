// The callers of the projection step (include/orchard_b200_cases.h): the
// Taylor-Green and lid-driven-cavity drivers with their config files and
// validation gates, the SLVCHKP1 checkpoint and the legacy-VTK export.
//
// Everything here is host code over the step ABI of orchard_b200.h: a case
// context is an of_ctx on the case grid, the state stays resident on the
// device between calls, and only diagnostics, centreline lines and the fields
// a file needs cross PCIe.  Texts, number formatting and file bytes follow
// the reference, since its tests and harness scripts parse them.
#include "../../include/orchard_b200_cases.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace ofb {
void set_last_error(const std::string& message);
}

namespace {

// ---------------------------------------------------------------------------
// Errors: a failing step-ABI call keeps its status and text; everything else
// maps like the step ABI (invalid_argument / out_of_range -> INVALID_ARGUMENT,
// other exceptions -> RUNTIME_ERROR).
// ---------------------------------------------------------------------------

struct Failure : std::runtime_error {
  of_status status;
  Failure(of_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void check(of_status s) {
  if(s != OF_OK) throw Failure(s, of_last_error());
}

template <typename Fn>
of_status guarded(Fn&& fn) {
  try {
    fn();
    ofb::set_last_error("");
    return OF_OK;
  } catch(const Failure& e) {
    ofb::set_last_error(e.what());
    return e.status;
  } catch(const std::invalid_argument& e) {
    ofb::set_last_error(e.what());
    return OF_INVALID_ARGUMENT;
  } catch(const std::out_of_range& e) {
    ofb::set_last_error(e.what());
    return OF_INVALID_ARGUMENT;
  } catch(const std::exception& e) {
    ofb::set_last_error(e.what());
    return OF_RUNTIME_ERROR;
  }
}

void need(const void* p, const char* what) {
  if(p == nullptr) throw std::invalid_argument(std::string(what) + " must not be null");
}

void copy_text(char* dst, size_t cap, const std::string& s) {
  if(cap == 0) return;
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(dst, s.data(), n);
  dst[n] = '\0';
}

// ---------------------------------------------------------------------------
// Config files: `key = value`, '#' starts a comment, blank lines skipped
// (solver/taylor_green.cpp:425-481, solver/lid_driven_cavity.cpp:296-336).
// ---------------------------------------------------------------------------

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if(a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

bool parse_bool(const std::string& v) {
  static const char* yes[] = {"true", "1", "yes", "on"};
  static const char* no[] = {"false", "0", "no", "off"};
  for(const char* t : yes)
    if(v == t) return true;
  for(const char* t : no)
    if(v == t) return false;
  throw std::runtime_error("invalid boolean value: " + v);
}

// Calls on_entry(key, value) for every setting of the file.
void read_settings(const std::string& path, const std::string& what,
                   const std::function<void(const std::string&, const std::string&)>& on_entry) {
  std::ifstream in(path);
  if(!in.is_open()) throw std::runtime_error("unable to open " + what + " config: " + path);
  std::string line;
  int number = 0;
  while(std::getline(in, line)) {
    ++number;
    const size_t hash = line.find('#');
    if(hash != std::string::npos) line.resize(hash);
    line = trim(line);
    if(line.empty()) continue;
    const size_t eq = line.find('=');
    if(eq == std::string::npos)
      throw std::runtime_error("invalid config line " + std::to_string(number) + ": " + line);
    on_entry(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
  }
}

std::string scheme_name(int scheme) {
  switch(scheme) {
    case OF_ADVECTION_TVD: return "tvd";
    case OF_ADVECTION_UPWIND: return "upwind";
    case OF_ADVECTION_CENTRAL: return "central";
    default: return "unknown";
  }
}

std::string limiter_name(int limiter) { return limiter == OF_LIMITER_VAN_LEER ? "van_leer" : "unknown"; }

std::string advection_text(int scheme, int limiter) {
  return "scheme=" + scheme_name(scheme) + ", limiter=" + limiter_name(limiter);
}

std::string backend_name(int backend) {
  switch(backend) {
    case OF_BACKEND_CPU: return "cpu";
    case OF_BACKEND_METAL: return "metal";
    default: return "unknown";
  }
}

// The step implements the TVD / van Leer advection only.
void require_step_scheme(int scheme, int limiter) {
  if(scheme != OF_ADVECTION_TVD || limiter != OF_LIMITER_VAN_LEER)
    throw std::invalid_argument("the B200 step implements the tvd scheme with the van_leer limiter only");
}

of_face_bc face(int type) {
  of_face_bc f{};
  f.type = type;
  return f;
}

// ---------------------------------------------------------------------------
// Taylor-Green case (solver/taylor_green.cpp)
// ---------------------------------------------------------------------------

void validate_tg(const of_tg_config& c) {
  if(c.nx <= 0 || c.ny <= 0 || c.nz <= 0)
    throw std::invalid_argument("Taylor-Green config expects positive nx, ny, and nz");
  if(c.viscosity <= 0.0) throw std::invalid_argument("Taylor-Green config expects viscosity > 0");
  if(c.cfl_limit <= 0.0) throw std::invalid_argument("Taylor-Green config expects cfl_limit > 0");
  if(c.final_time <= 0.0) throw std::invalid_argument("Taylor-Green config expects final_time > 0");
  if(c.poisson_max_iterations <= 0 || c.poisson_tolerance <= 0.0)
    throw std::invalid_argument("Taylor-Green config expects positive Poisson controls");
}

bool tg_3d(const of_tg_config& c) { return c.nz > 1; }

of_tg_config tg_default() {
  of_tg_config c{};
  c.nx = 128;
  c.ny = 128;
  c.nz = 1;
  c.viscosity = 0.01;
  c.cfl_limit = 0.5;
  c.final_time = 0.5;
  c.poisson_max_iterations = 200;
  c.poisson_tolerance = 1.0e-10;
  c.validate_energy = 1;
  c.backend = OF_BACKEND_CPU;
  c.advection_scheme = OF_ADVECTION_TVD;
  c.advection_limiter = OF_LIMITER_VAN_LEER;
  return c;
}

of_grid tg_grid(const of_tg_config& c) {
  validate_tg(c);
  const double length = 2.0 * std::acos(-1.0);
  return of_grid{c.nx, c.ny, c.nz, length / c.nx, length / c.ny, tg_3d(c) ? length / c.nz : 1.0};
}

of_bc tg_bc(const of_tg_config& c) {
  of_bc bc{};
  for(int f = 0; f < 6; ++f) bc.faces[f] = face(OF_PERIODIC);
  if(!tg_3d(c)) bc.faces[4] = bc.faces[5] = face(OF_SYMMETRY);
  return bc;
}

// taylor_green_dt: final_time split into ceil(final_time / dt_max) equal steps,
// dt_max = cfl / (1/dx + 1/dy [+ 1/dz]).
double tg_dt(const of_tg_config& c) {
  const of_grid g = tg_grid(c);
  const double inv = 1.0 / g.dx + 1.0 / g.dy + (g.nz == 1 ? 0.0 : 1.0 / g.dz);
  const double upper = c.cfl_limit / inv;
  const int steps = std::max(1, static_cast<int>(std::ceil(c.final_time / upper)));
  return c.final_time / static_cast<double>(steps);
}

// Steps run_taylor_green takes: ceil(final_time / dt) with dt as above.
int tg_steps(const of_tg_config& c) { return static_cast<int>(std::ceil(c.final_time / tg_dt(c))); }

std::string tg_describe(const of_tg_config& c) {
  std::ostringstream o;
  o << "nx=" << c.nx << ", ny=" << c.ny << ", nz=" << c.nz << ", viscosity=" << c.viscosity
    << ", cfl_limit=" << c.cfl_limit << ", final_time=" << c.final_time
    << ", poisson_max_iterations=" << c.poisson_max_iterations
    << ", poisson_tolerance=" << c.poisson_tolerance
    << ", validate_energy=" << (c.validate_energy ? "true" : "false")
    << ", backend=" << backend_name(c.backend)
    << ", advection=" << advection_text(c.advection_scheme, c.advection_limiter);
  return o.str();
}

of_step_params tg_params(const of_tg_config& c) {
  of_step_params p{};
  p.viscosity = c.viscosity;
  p.dt = tg_dt(c);
  p.density = 1.0;
  p.poisson_max_iterations = c.poisson_max_iterations;
  p.poisson_tolerance = c.poisson_tolerance;
  p.correction_variant = OF_CORRECTION_TAYLOR_GREEN;
  p.track_max_divergence = 1;
  p.solver_name = "Taylor-Green";
  return p;
}

bool same_grid(const of_grid& a, const of_grid& b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.dx == b.dx && a.dy == b.dy && a.dz == b.dz;
}

of_grid ctx_grid(of_ctx* ctx) {
  need(ctx, "context");
  of_grid g{};
  check(of_get_grid(ctx, &g));
  return g;
}

of_step_metrics ctx_metrics(of_ctx* ctx) {
  of_step_metrics m{};
  int has_prev = 0;
  check(of_state_download(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &has_prev, &m));
  return m;
}

void require_tg_state(of_ctx* ctx, const of_tg_config& c) {
  if(!same_grid(ctx_grid(ctx), tg_grid(c)))
    throw std::invalid_argument("Taylor-Green state grid does not match the config");
}

std::string device_name() {
  int dev = 0;
  cudaDeviceProp prop{};
  if(cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
    return "cuda";
  return prop.name;
}

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

// ---------------------------------------------------------------------------
// Lid-driven cavity case (solver/lid_driven_cavity.cpp)
// ---------------------------------------------------------------------------

void validate_cavity(const of_cavity_config& c) {
  if(c.nx <= 0 || c.ny <= 0) throw std::invalid_argument("lid-driven cavity config expects positive nx and ny");
  if(c.reynolds <= 0.0) throw std::invalid_argument("lid-driven cavity config expects reynolds > 0");
  if(c.lid_velocity <= 0.0) throw std::invalid_argument("lid-driven cavity config expects lid_velocity > 0");
  if(c.cfl_limit <= 0.0) throw std::invalid_argument("lid-driven cavity config expects cfl_limit > 0");
  if(c.max_steps <= 0 || c.min_steps < 0)
    throw std::invalid_argument("lid-driven cavity config expects non-negative step controls");
  if(c.poisson_max_iterations <= 0 || c.poisson_tolerance <= 0.0)
    throw std::invalid_argument("lid-driven cavity config expects positive Poisson controls");
}

of_cavity_config cavity_default() {
  of_cavity_config c{};
  c.nx = 128;
  c.ny = 128;
  c.reynolds = 100.0;
  c.lid_velocity = 1.0;
  c.cfl_limit = 0.5;
  c.max_steps = 8000;
  c.min_steps = 200;
  c.steady_tolerance = 1.0e-7;
  c.poisson_max_iterations = 200;
  c.poisson_tolerance = 1.0e-10;
  c.validate_reference = 1;
  c.advection_scheme = OF_ADVECTION_TVD;
  c.advection_limiter = OF_LIMITER_VAN_LEER;
  return c;
}

of_grid cavity_grid(const of_cavity_config& c) {
  return of_grid{c.nx, c.ny, 1, 1.0 / c.nx, 1.0 / c.ny, 1.0};
}

// No-slip walls, the lid moving with (U, 0, 0) on y_max, symmetry in z.
of_bc cavity_bc(const of_cavity_config& c) {
  of_bc bc{};
  for(int f = 0; f < 6; ++f) bc.faces[f] = face(OF_NO_SLIP_WALL);
  bc.faces[3] = face(OF_PRESCRIBED_VELOCITY);
  bc.faces[3].velocity[0] = c.lid_velocity;
  bc.faces[4] = bc.faces[5] = face(OF_SYMMETRY);
  return bc;
}

double cavity_viscosity(const of_cavity_config& c) { return c.lid_velocity / c.reynolds; }

double cavity_dt(const of_cavity_config& c) {
  const of_grid g = cavity_grid(c);
  return c.cfl_limit / (c.lid_velocity / g.dx + c.lid_velocity / g.dy);
}

std::string cavity_describe(const of_cavity_config& c) {
  std::ostringstream o;
  o << "nx=" << c.nx << ", ny=" << c.ny << ", Re=" << c.reynolds << ", lid_velocity=" << c.lid_velocity
    << ", cfl_limit=" << c.cfl_limit << ", max_steps=" << c.max_steps << ", min_steps=" << c.min_steps
    << ", steady_tolerance=" << c.steady_tolerance
    << ", poisson_max_iterations=" << c.poisson_max_iterations
    << ", poisson_tolerance=" << c.poisson_tolerance
    << ", validate_reference=" << (c.validate_reference ? "true" : "false")
    << ", advection=" << advection_text(c.advection_scheme, c.advection_limiter);
  return o.str();
}

of_step_params cavity_params(const of_cavity_config& c) {
  of_step_params p{};
  p.viscosity = cavity_viscosity(c);
  p.dt = cavity_dt(c);
  p.density = 1.0;
  p.poisson_max_iterations = c.poisson_max_iterations;
  p.poisson_tolerance = c.poisson_tolerance;
  p.correction_variant = OF_CORRECTION_CAVITY;
  p.track_max_divergence = 0;
  p.solver_name = "lid-driven cavity";
  return p;
}

void require_cavity_state(of_ctx* ctx, const of_cavity_config& c) {
  validate_cavity(c);
  if(!same_grid(ctx_grid(ctx), cavity_grid(c)))
    throw std::invalid_argument("lid-driven cavity state grid does not match the config");
}

bool steady(const of_cavity_config& c, const of_step_metrics& m) {
  return m.step >= c.min_steps && m.max_velocity_change <= c.steady_tolerance;
}

struct Profile {
  std::vector<double> x, v;
};

// Centreline profiles (solver/lid_driven_cavity.cpp:100-131): u through the
// middle u-face column i = 1 + (nx + 1) / 2, v through the middle v-face row
// j = 1 + (ny + 1) / 2, active entries of the first k plane.  The resident
// velocity already carries its ghost fills, and the fills leave these
// interior entries unchanged.
void centerlines(of_ctx* ctx, Profile& pu, Profile& pv) {
  const of_grid g = ctx_grid(ctx);
  std::vector<double> line(static_cast<size_t>(std::max(g.nx, g.ny)) + 3);
  int n = 0;
  const int ic = 1 + (g.nx + 1) / 2;
  check(of_sample_line(ctx, 1, 1, ic, 0, 1, line.data(), &n));
  pu.x.resize(g.ny);
  pu.v.resize(g.ny);
  for(int j = 1; j <= g.ny; ++j) {
    pu.x[j - 1] = (static_cast<double>(j - 1) + 0.5) * g.dy;
    pu.v[j - 1] = line[j];
  }
  const int jc = 1 + (g.ny + 1) / 2;
  check(of_sample_line(ctx, 2, 0, 0, jc, 1, line.data(), &n));
  pv.x.resize(g.nx);
  pv.v.resize(g.nx);
  for(int i = 1; i <= g.nx; ++i) {
    pv.x[i - 1] = (static_cast<double>(i - 1) + 0.5) * g.dx;
    pv.v[i - 1] = line[i];
  }
}

// Value of a sampled profile at `at`: the sample itself on a node, else the
// cubic through the four nodes around the bracket (clamped to the ends), or
// the chord for profiles of fewer than four samples
// (interpolate_profile_value, solver/lid_driven_cavity.cpp:191-232).
double profile_at(const Profile& p, double at) {
  const size_t n = p.x.size();
  if(n != p.v.size() || n < 2)
    throw std::invalid_argument("centerline profile interpolation requires matching sample arrays");
  if(at < p.x.front() || at > p.x.back())
    throw std::out_of_range("reference coordinate falls outside the sampled centerline range");
  const size_t hi = static_cast<size_t>(std::lower_bound(p.x.begin(), p.x.end(), at) - p.x.begin());
  if(hi == 0) return p.v.front();
  if(hi == n) return p.v.back();
  if(p.x[hi] == at) return p.v[hi];
  const size_t lo = hi - 1;
  if(n >= 4) {
    const size_t first = std::min(lo > 0 ? lo - 1 : 0, n - 4);
    double sum = 0.0;
    for(size_t a = first; a < first + 4; ++a) {
      double w = 1.0;
      for(size_t b = first; b < first + 4; ++b)
        if(b != a) w *= (at - p.x[b]) / (p.x[a] - p.x[b]);
      sum += w * p.v[a];
    }
    return sum;
  }
  const double t = (at - p.x[lo]) / (p.x[hi] - p.x[lo]);
  return (1.0 - t) * p.v[lo] + t * p.v[hi];
}

// Relative distance of a sample to the envelope [lo, hi] (0 inside).
double envelope_miss(double value, double lo, double hi) {
  const double a = std::min(lo, hi), b = std::max(lo, hi);
  if(value >= a && value <= b) return 0.0;
  const double nearest = value < a ? a : b;
  return std::abs(value - nearest) / std::abs(nearest);
}

struct EnvelopePoint {
  const char* label;
  int line;
  double coordinate, value, lower, upper;
};

// The Re 100 centreline envelope of the reference's gate
// (re100_centerline_reference_envelope, solver/lid_driven_cavity.cpp:410-443).
constexpr const char* kEnvelopeDataset = "Re100_centerline_literature_envelope";
constexpr EnvelopePoint kEnvelope[4] = {
    {"u_vertical_y0.9766", OF_U_VERTICAL, 0.9766, 0.84123, 0.84123, 0.84123},
    {"u_vertical_y0.4531", OF_U_VERTICAL, 0.4531, -0.21090, -0.21400, -0.21060},
    {"v_horizontal_x0.2344", OF_V_HORIZONTAL, 0.2344, 0.17527, 0.17527, 0.17960},
    {"v_horizontal_x0.8047", OF_V_HORIZONTAL, 0.8047, -0.24533, -0.25400, -0.24533},
};

// ---------------------------------------------------------------------------
// SLVCHKP1 (io/checkpoint.cpp): "SLVCHKP1", u32 version 1, u64 payload bytes,
// u64 FNV-1a of the payload, then tagged sections (4-byte tag, u64 size,
// bytes), all little-endian.  Fields: u32 storage extents, then the padded
// storage in k-j-i order, i.e. the storage array itself.
// ---------------------------------------------------------------------------

constexpr uint64_t kFnvOffset = 14695981039346656037ull;
constexpr uint64_t kFnvPrime = 1099511628211ull;

uint64_t fnv_update(uint64_t h, const uint8_t* p, size_t n) {
  for(size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= kFnvPrime;
  }
  return h;
}

uint64_t fnv_text(const std::string& s) {
  return fnv_update(kFnvOffset, reinterpret_cast<const uint8_t*>(s.data()), s.size());
}

struct Out {
  std::vector<uint8_t> b;
  void u32(uint32_t v) {
    for(int s = 0; s < 32; s += 8) b.push_back(static_cast<uint8_t>(v >> s));
  }
  void u64(uint64_t v) {
    for(int s = 0; s < 64; s += 8) b.push_back(static_cast<uint8_t>(v >> s));
  }
  void f64(double v) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    u64(u);
  }
};

struct In {
  const uint8_t* p;
  size_t n;
  size_t at = 0;
  uint32_t u32() {
    if(at + 4 > n) throw std::runtime_error("checkpoint truncated while reading u32");
    uint32_t v = 0;
    for(int s = 0; s < 32; s += 8) v |= static_cast<uint32_t>(p[at++]) << s;
    return v;
  }
  uint64_t u64() {
    if(at + 8 > n) throw std::runtime_error("checkpoint truncated while reading u64");
    uint64_t v = 0;
    for(int s = 0; s < 64; s += 8) v |= static_cast<uint64_t>(p[at++]) << s;
    return v;
  }
  double f64() {
    const uint64_t u = u64();
    double v;
    std::memcpy(&v, &u, 8);
    return v;
  }
};

constexpr char kMagic[8] = {'S', 'L', 'V', 'C', 'H', 'K', 'P', '1'};
constexpr uint32_t kFormatVersion = 1;

// The state a checkpoint carries, in host memory.
struct HostState {
  of_grid grid{};
  std::array<std::vector<double>, 7> f;  // u, v, w, adv_u, adv_v, adv_w, p_total
  int has_prev = 0;
  of_step_metrics metrics{};
};

constexpr const char* kFieldTags[7] = {"VELX", "VELY", "VELZ", "ADVX", "ADVY", "ADVZ", "PRST"};

// Storage extents of field f (0..6) on grid g.
std::array<int, 3> storage(const of_grid& g, int f) {
  const int loc = f == 6 ? 0 : 1 + f % 3;
  return {g.nx + 2 + (loc == 1), g.ny + 2 + (loc == 2), g.nz + 2 + (loc == 3)};
}

size_t storage_count(const of_grid& g, int f) {
  const auto e = storage(g, f);
  return static_cast<size_t>(e[0]) * e[1] * e[2];
}

std::vector<uint8_t> meta_bytes(uint64_t build_hash, uint64_t config_hash, const HostState& s) {
  Out o;
  o.u32(static_cast<uint32_t>(sizeof(double)));
  o.u64(build_hash);
  o.u64(config_hash);
  o.u32(s.has_prev ? 1u : 0u);
  o.u32(static_cast<uint32_t>(s.metrics.step));
  o.f64(s.metrics.time);
  o.f64(s.metrics.dt);
  o.f64(s.metrics.max_cfl);
  o.f64(s.metrics.max_velocity_change);
  o.f64(s.metrics.divergence_l2);
  o.u32(static_cast<uint32_t>(s.metrics.pressure_iterations));
  o.f64(s.metrics.pressure_relative_residual);
  return o.b;
}

std::vector<uint8_t> grid_bytes(const of_grid& g) {
  Out o;
  o.u32(static_cast<uint32_t>(g.nx));
  o.u32(static_cast<uint32_t>(g.ny));
  o.u32(static_cast<uint32_t>(g.nz));
  o.f64(g.dx);
  o.f64(g.dy);
  o.f64(g.dz);
  o.u32(1u);  // ghost layers
  return o.b;
}

std::vector<uint8_t> cavity_config_bytes(const of_cavity_config& c) {
  Out o;
  o.u32(static_cast<uint32_t>(c.nx));
  o.u32(static_cast<uint32_t>(c.ny));
  o.f64(c.reynolds);
  o.f64(c.lid_velocity);
  o.f64(c.cfl_limit);
  o.u32(static_cast<uint32_t>(c.max_steps));
  o.u32(static_cast<uint32_t>(c.min_steps));
  o.f64(c.steady_tolerance);
  o.u32(static_cast<uint32_t>(c.poisson_max_iterations));
  o.f64(c.poisson_tolerance);
  o.u32(c.validate_reference ? 1u : 0u);
  o.u32(static_cast<uint32_t>(c.advection_scheme));
  o.u32(static_cast<uint32_t>(c.advection_limiter));
  return o.b;
}

std::vector<uint8_t> tg_config_bytes(const of_tg_config& c) {
  Out o;
  o.u32(static_cast<uint32_t>(c.nx));
  o.u32(static_cast<uint32_t>(c.ny));
  o.u32(static_cast<uint32_t>(c.nz));
  o.f64(c.viscosity);
  o.f64(c.cfl_limit);
  o.f64(c.final_time);
  o.u32(static_cast<uint32_t>(c.poisson_max_iterations));
  o.f64(c.poisson_tolerance);
  o.u32(c.validate_energy ? 1u : 0u);
  o.u32(static_cast<uint32_t>(c.backend));
  o.u32(static_cast<uint32_t>(c.advection_scheme));
  o.u32(static_cast<uint32_t>(c.advection_limiter));
  return o.b;
}

// Streams the file: a placeholder header, the sections (hashed on the way),
// then the real header written over the placeholder.  Bytes equal those of
// write_lid_driven_cavity_checkpoint (io/checkpoint.cpp:313-349).
class Writer {
 public:
  explicit Writer(const std::string& path) : path_(path), out_(path, std::ios::binary) {
    if(!out_.is_open()) throw std::runtime_error("unable to open checkpoint for writing: " + path);
    out_.write(kMagic, 8);
    const uint8_t zeros[20] = {};
    out_.write(reinterpret_cast<const char*>(zeros), sizeof(zeros));
  }
  void section(const char* tag, const std::vector<uint8_t>& body) {
    header(tag, body.size());
    put(body.data(), body.size());
  }
  void field(const char* tag, const of_grid& g, int f, const std::vector<double>& data) {
    const auto e = storage(g, f);
    Out o;
    for(int a = 0; a < 3; ++a) o.u32(static_cast<uint32_t>(e[a]));
    header(tag, o.b.size() + data.size() * sizeof(double));
    put(o.b.data(), o.b.size());
    static_assert(sizeof(double) == 8, "IEEE double");
    put(reinterpret_cast<const uint8_t*>(data.data()), data.size() * sizeof(double));
  }
  void finish() {
    Out h;
    h.u32(kFormatVersion);
    h.u64(size_);
    h.u64(hash_);
    out_.seekp(8);
    out_.write(reinterpret_cast<const char*>(h.b.data()), static_cast<std::streamsize>(h.b.size()));
    out_.flush();
    if(!out_.good()) throw std::runtime_error("failed while writing checkpoint: " + path_);
  }

 private:
  void header(const char* tag, uint64_t n) {
    Out o;
    for(int i = 0; i < 4; ++i) o.b.push_back(static_cast<uint8_t>(tag[i]));
    o.u64(n);
    put(o.b.data(), o.b.size());
  }
  void put(const uint8_t* p, size_t n) {
    hash_ = fnv_update(hash_, p, n);
    size_ += n;
    out_.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n));
  }
  std::string path_;
  std::ofstream out_;
  uint64_t hash_ = kFnvOffset;
  uint64_t size_ = 0;
};

void write_checkpoint(const std::string& path, uint64_t build_hash, uint64_t config_hash,
                      const char* config_tag, const std::vector<uint8_t>& config, const HostState& s,
                      bool with_max_divergence) {
  Writer w(path);
  w.section("META", meta_bytes(build_hash, config_hash, s));
  w.section(config_tag, config);
  w.section("GRID", grid_bytes(s.grid));
  for(int f = 0; f < 7; ++f) w.field(kFieldTags[f], s.grid, f, s.f[f]);
  if(with_max_divergence) {
    Out o;
    o.f64(s.metrics.max_divergence_l2);
    w.section("MDIV", o.b);
  }
  w.finish();
}

std::vector<uint8_t> read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if(!in.is_open()) throw std::runtime_error("unable to open checkpoint: " + path);
  in.seekg(0, std::ios::end);
  const std::streamsize n = in.tellg();
  in.seekg(0, std::ios::beg);
  if(n < 0) throw std::runtime_error("unable to read checkpoint size: " + path);
  std::vector<uint8_t> b(static_cast<size_t>(n));
  if(!in.read(reinterpret_cast<char*>(b.data()), n))
    throw std::runtime_error("unable to read checkpoint payload: " + path);
  return b;
}

// What a load checks a file against.
struct Expect {
  uint64_t build_hash;
  uint64_t config_hash;
  const char* config_tag;
  std::function<void(In&)> check_config;  // parses and compares the config section
  of_grid grid;
  bool with_max_divergence;
};

bool tag_is(const uint8_t* p, const char* tag) { return std::memcmp(p, tag, 4) == 0; }

// load_lid_driven_cavity_checkpoint (io/checkpoint.cpp:351-461): every check,
// in file order, before the state is handed out.
HostState load_checkpoint(const std::string& path, const Expect& x, of_checkpoint_meta& meta) {
  const std::vector<uint8_t> bytes = read_file(path);
  if(bytes.size() < 8 + 4 + 8 + 8) throw std::runtime_error("checkpoint file is too small: " + path);
  if(std::memcmp(bytes.data(), kMagic, 8) != 0) throw std::runtime_error("checkpoint magic mismatch: " + path);
  In head{bytes.data(), bytes.size(), 8};
  const uint32_t version = head.u32();
  if(version != kFormatVersion)
    throw std::runtime_error("unsupported checkpoint format version: " + std::to_string(version));
  const uint64_t payload = head.u64();
  const uint64_t checksum = head.u64();
  const size_t start = head.at;
  if(start + payload != bytes.size())
    throw std::runtime_error("checkpoint payload length does not match the file size");
  if(fnv_update(kFnvOffset, bytes.data() + start, static_cast<size_t>(payload)) != checksum)
    throw std::runtime_error("checkpoint checksum verification failed");

  HostState s;
  s.grid = x.grid;
  meta = of_checkpoint_meta{};
  meta.format_version = version;
  meta.checksum = checksum;
  bool have_meta = false, have_config = false, have_grid = false, have_mdiv = false;
  std::array<bool, 7> have_field{};

  size_t at = start;
  while(at < bytes.size()) {
    if(at + 12 > bytes.size()) throw std::runtime_error("checkpoint section header is truncated");
    const uint8_t* tag = bytes.data() + at;
    In sz{bytes.data(), bytes.size(), at + 4};
    const uint64_t n = sz.u64();
    at += 12;
    if(at + n > bytes.size()) throw std::runtime_error("checkpoint section payload is truncated");
    In sec{bytes.data() + at, static_cast<size_t>(n), 0};
    at += static_cast<size_t>(n);

    if(tag_is(tag, "META")) {
      meta.scalar_bytes = sec.u32();
      meta.build_hash = sec.u64();
      meta.configuration_hash = sec.u64();
      s.has_prev = sec.u32() != 0u;
      s.metrics.step = static_cast<int>(sec.u32());
      s.metrics.time = sec.f64();
      s.metrics.dt = sec.f64();
      s.metrics.max_cfl = sec.f64();
      s.metrics.max_velocity_change = sec.f64();
      s.metrics.divergence_l2 = sec.f64();
      s.metrics.pressure_iterations = static_cast<int>(sec.u32());
      s.metrics.pressure_relative_residual = sec.f64();
      if(sec.at != sec.n) throw std::runtime_error("checkpoint metadata section contains trailing bytes");
      if(meta.scalar_bytes != sizeof(double))
        throw std::runtime_error("checkpoint precision does not match the current solver precision");
      if(meta.build_hash != x.build_hash)
        throw std::runtime_error("checkpoint build hash does not match the current executable");
      if(meta.configuration_hash != x.config_hash)
        throw std::runtime_error("checkpoint configuration hash does not match the requested config");
      have_meta = true;
    } else if(tag_is(tag, x.config_tag)) {
      x.check_config(sec);
      have_config = true;
    } else if(tag_is(tag, "GRID")) {
      of_grid g{};
      g.nx = static_cast<int>(sec.u32());
      g.ny = static_cast<int>(sec.u32());
      g.nz = static_cast<int>(sec.u32());
      g.dx = sec.f64();
      g.dy = sec.f64();
      g.dz = sec.f64();
      const int ghosts = static_cast<int>(sec.u32());
      if(sec.at != sec.n) throw std::runtime_error("checkpoint grid section contains trailing bytes");
      if(!same_grid(g, x.grid) || ghosts != 1)
        throw std::runtime_error("checkpoint grid does not match the requested run configuration");
      have_grid = true;
    } else if(x.with_max_divergence && tag_is(tag, "MDIV")) {
      s.metrics.max_divergence_l2 = sec.f64();
      if(sec.at != sec.n) throw std::runtime_error("checkpoint metadata section contains trailing bytes");
      have_mdiv = true;
    } else {
      for(int f = 0; f < 7; ++f) {
        if(!tag_is(tag, kFieldTags[f])) continue;
        const auto e = storage(x.grid, f);
        const int ex = static_cast<int>(sec.u32()), ey = static_cast<int>(sec.u32()),
                  ez = static_cast<int>(sec.u32());
        if(ex != e[0] || ey != e[1] || ez != e[2])
          throw std::runtime_error("checkpoint field extent does not match the current layout");
        const size_t count = storage_count(x.grid, f);
        if(sec.n - sec.at < count * sizeof(double))
          throw std::runtime_error("checkpoint truncated while reading u64");
        s.f[f].resize(count);
        std::memcpy(s.f[f].data(), sec.p + sec.at, count * sizeof(double));
        sec.at += count * sizeof(double);
        if(sec.at != sec.n) throw std::runtime_error("checkpoint field section contains trailing bytes");
        have_field[f] = true;
      }
    }
  }
  bool complete = have_meta && have_config && have_grid && (!x.with_max_divergence || have_mdiv);
  for(bool h : have_field) complete = complete && h;
  if(!complete) throw std::runtime_error("checkpoint is missing one or more required sections");
  return s;
}

Expect cavity_expect(const of_cavity_config& c, uint64_t build_hash) {
  Expect x;
  x.build_hash = build_hash;
  x.config_hash = fnv_text(cavity_describe(c));
  x.config_tag = "CONF";
  x.check_config = [c](In& in) {
    of_cavity_config l{};
    l.nx = static_cast<int>(in.u32());
    l.ny = static_cast<int>(in.u32());
    l.reynolds = in.f64();
    l.lid_velocity = in.f64();
    l.cfl_limit = in.f64();
    l.max_steps = static_cast<int>(in.u32());
    l.min_steps = static_cast<int>(in.u32());
    l.steady_tolerance = in.f64();
    l.poisson_max_iterations = static_cast<int>(in.u32());
    l.poisson_tolerance = in.f64();
    l.validate_reference = in.u32() != 0u;
    l.advection_scheme = static_cast<int>(in.u32());
    l.advection_limiter = static_cast<int>(in.u32());
    if(in.at != in.n) throw std::runtime_error("checkpoint config section contains trailing bytes");
    if(l.nx != c.nx || l.ny != c.ny || l.reynolds != c.reynolds || l.lid_velocity != c.lid_velocity ||
       l.cfl_limit != c.cfl_limit || l.max_steps != c.max_steps || l.min_steps != c.min_steps ||
       l.steady_tolerance != c.steady_tolerance || l.poisson_max_iterations != c.poisson_max_iterations ||
       l.poisson_tolerance != c.poisson_tolerance || l.validate_reference != (c.validate_reference != 0) ||
       l.advection_scheme != c.advection_scheme || l.advection_limiter != c.advection_limiter)
      throw std::runtime_error("checkpoint config does not match the requested run configuration");
  };
  x.grid = cavity_grid(c);
  x.with_max_divergence = false;
  return x;
}

Expect tg_expect(const of_tg_config& c, uint64_t build_hash) {
  Expect x;
  x.build_hash = build_hash;
  x.config_hash = fnv_text(tg_describe(c));
  x.config_tag = "TGCF";
  x.check_config = [c](In& in) {
    of_tg_config l{};
    l.nx = static_cast<int>(in.u32());
    l.ny = static_cast<int>(in.u32());
    l.nz = static_cast<int>(in.u32());
    l.viscosity = in.f64();
    l.cfl_limit = in.f64();
    l.final_time = in.f64();
    l.poisson_max_iterations = static_cast<int>(in.u32());
    l.poisson_tolerance = in.f64();
    l.validate_energy = in.u32() != 0u;
    l.backend = static_cast<int>(in.u32());
    l.advection_scheme = static_cast<int>(in.u32());
    l.advection_limiter = static_cast<int>(in.u32());
    if(in.at != in.n) throw std::runtime_error("checkpoint config section contains trailing bytes");
    if(l.nx != c.nx || l.ny != c.ny || l.nz != c.nz || l.viscosity != c.viscosity ||
       l.cfl_limit != c.cfl_limit || l.final_time != c.final_time ||
       l.poisson_max_iterations != c.poisson_max_iterations || l.poisson_tolerance != c.poisson_tolerance ||
       l.validate_energy != (c.validate_energy != 0) || l.backend != c.backend ||
       l.advection_scheme != c.advection_scheme || l.advection_limiter != c.advection_limiter)
      throw std::runtime_error("checkpoint config does not match the requested run configuration");
  };
  x.grid = tg_grid(c);
  x.with_max_divergence = true;
  return x;
}

// Build description of this library: project, version, the CUDA runtime it
// was built against, the deterministic profile, no fast-math.
uint64_t library_build_hash() {
  const std::string version =
      std::to_string(CUDART_VERSION / 1000) + "." + std::to_string(CUDART_VERSION % 1000 / 10);
  return of_build_hash("Orchard Flow B200", "0.1.0", "NVIDIA CUDA", version.c_str(), "deterministic", 0);
}

uint64_t resolve_hash(uint64_t h) { return h != 0 ? h : library_build_hash(); }

HostState download_state(of_ctx* ctx) {
  HostState s;
  s.grid = ctx_grid(ctx);
  for(int f = 0; f < 7; ++f) s.f[f].resize(storage_count(s.grid, f));
  check(of_state_download(ctx, s.f[0].data(), s.f[1].data(), s.f[2].data(), s.f[3].data(), s.f[4].data(),
                          s.f[5].data(), s.f[6].data(), &s.has_prev, &s.metrics));
  return s;
}

void upload_state(of_ctx* ctx, const HostState& s) {
  check(of_state_upload(ctx, s.f[0].data(), s.f[1].data(), s.f[2].data(), s.f[3].data(), s.f[4].data(),
                        s.f[5].data(), s.f[6].data(), s.has_prev, &s.metrics));
}

HostState host_state(const of_grid& g, const double* const* f, int has_prev, const of_step_metrics* m) {
  HostState s;
  s.grid = g;
  for(int i = 0; i < 7; ++i) {
    need(f[i], "state field");
    s.f[i].assign(f[i], f[i] + storage_count(g, i));
  }
  s.has_prev = has_prev ? 1 : 0;
  if(m) s.metrics = *m;
  return s;
}

// %g with six significant digits: the default formatting of a double on a
// std::ostream, which the reference's VTK writer and reports use.
void put_number(std::FILE* f, double v) { std::fprintf(f, "%g", v); }

}  // namespace

extern "C" {

// ---- Taylor-Green ---------------------------------------------------------

of_status of_tg_config_default(of_tg_config* config) {
  return guarded([&] {
    need(config, "config");
    *config = tg_default();
  });
}

of_status of_tg_config_load(const char* path, of_tg_config* config) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    of_tg_config c = tg_default();
    read_settings(path, "Taylor-Green", [&](const std::string& k, const std::string& v) {
      if(k == "nx") c.nx = std::stoi(v);
      else if(k == "ny") c.ny = std::stoi(v);
      else if(k == "nz") c.nz = std::stoi(v);
      else if(k == "viscosity") c.viscosity = std::stod(v);
      else if(k == "cfl_limit") c.cfl_limit = std::stod(v);
      else if(k == "final_time") c.final_time = std::stod(v);
      else if(k == "poisson_max_iterations") c.poisson_max_iterations = std::stoi(v);
      else if(k == "poisson_tolerance") c.poisson_tolerance = std::stod(v);
      else if(k == "validate_energy") c.validate_energy = parse_bool(v) ? 1 : 0;
      else if(k == "backend") {
        if(v == "cpu") c.backend = OF_BACKEND_CPU;
        else if(v == "metal") c.backend = OF_BACKEND_METAL;
        else throw std::runtime_error("invalid Taylor-Green backend value: " + v);
      } else throw std::runtime_error("unsupported Taylor-Green config key: " + k);
    });
    validate_tg(c);
    *config = c;
  });
}

of_status of_tg_config_describe(const of_tg_config* config, char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    need(config, "config");
    const std::string s = tg_describe(*config);
    if(buf) copy_text(buf, cap, s);
    if(len) *len = s.size();
  });
}

of_status of_tg_case(const of_tg_config* config, of_grid* grid, of_bc* bc, double* dt, int* steps) {
  return guarded([&] {
    need(config, "config");
    const of_grid g = tg_grid(*config);
    if(grid) *grid = g;
    if(bc) *bc = tg_bc(*config);
    if(dt) *dt = tg_dt(*config);
    if(steps) *steps = tg_steps(*config);
  });
}

of_status of_tg_create(const of_tg_config* config, int device, of_ctx** out) {
  return guarded([&] {
    need(config, "config");
    need(out, "output context pointer");
    *out = nullptr;
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    const of_grid g = tg_grid(*config);
    const of_bc bc = tg_bc(*config);
    of_ctx* ctx = nullptr;
    check(of_create(&g, &bc, device, &ctx));
    const of_status s = of_tg_init(ctx, config->viscosity, tg_dt(*config), 0);
    if(s != OF_OK) {
      const std::string msg = of_last_error();
      of_destroy(ctx);
      throw Failure(s, msg);
    }
    *out = ctx;
  });
}

of_status of_tg_run_steps(of_ctx* ctx, const of_tg_config* config, int steps, of_step_metrics* metrics) {
  return guarded([&] {
    need(config, "config");
    validate_tg(*config);
    if(steps < 0) throw std::invalid_argument("run_taylor_green_steps expects a non-negative step count");
    require_tg_state(ctx, *config);
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    const of_step_params p = tg_params(*config);
    check(of_run_steps(ctx, &p, steps, metrics));
  });
}

of_status of_tg_finalize(of_ctx* ctx, const of_tg_config* config, of_tg_result* result) {
  return guarded([&] {
    need(config, "config");
    need(result, "result");
    validate_tg(*config);
    require_tg_state(ctx, *config);
    of_tg_result r{};
    r.final_step = ctx_metrics(ctx);
    const bool three_d = tg_3d(*config);
    // exact_kinetic_energy (solver/taylor_green.cpp:263-267)
    const double e0 = three_d ? 0.125 : 0.25;
    const double rate = three_d ? 6.0 : 4.0;
    r.initial_kinetic_energy = e0 * std::exp(-rate * config->viscosity * 0.0);
    check(of_kinetic_energy(ctx, &r.final_kinetic_energy));
    if(config->validate_energy) {
      // build_validation (solver/taylor_green.cpp:403-417)
      const double exact = e0 * std::exp(-rate * config->viscosity * r.final_step.time);
      copy_text(r.reference_dataset, sizeof(r.reference_dataset),
                three_d ? "analytic_taylor_green_decay_3d" : "analytic_taylor_green_decay_2d");
      r.exact_kinetic_energy = exact;
      r.normalized_energy_error = std::abs(r.final_kinetic_energy - exact) / exact;
      check(of_tg_velocity_error(ctx, config->viscosity, r.final_step.time, 0, &r.velocity_relative_l2_error));
      r.pass = r.normalized_energy_error <= 1.0e-2 && r.final_step.divergence_l2 <= 1.0e-10;
    }
    copy_text(r.accelerator_name, sizeof(r.accelerator_name), device_name());
    *result = r;
  });
}

of_status of_tg_run(of_ctx* ctx, const of_tg_config* config, of_tg_result* result) {
  return guarded([&] {
    need(config, "config");
    need(result, "result");
    validate_tg(*config);
    if(config->backend == OF_BACKEND_METAL)
      throw std::runtime_error("the metal backend is not available: this build runs the step on a CUDA device");
    require_tg_state(ctx, *config);
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    check(of_tg_init(ctx, config->viscosity, tg_dt(*config), 0));
    const of_step_params p = tg_params(*config);
    const auto t0 = Clock::now();
    check(of_run_steps(ctx, &p, tg_steps(*config), nullptr));
    const double elapsed = seconds_since(t0);
    check(of_tg_finalize(ctx, config, result));
    result->elapsed_seconds = elapsed;
  });
}

// ---- lid-driven cavity ----------------------------------------------------

of_status of_cavity_config_default(of_cavity_config* config) {
  return guarded([&] {
    need(config, "config");
    *config = cavity_default();
  });
}

of_status of_cavity_config_load(const char* path, of_cavity_config* config) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    of_cavity_config c = cavity_default();
    read_settings(path, "cavity", [&](const std::string& k, const std::string& v) {
      if(k == "nx") c.nx = std::stoi(v);
      else if(k == "ny") c.ny = std::stoi(v);
      else if(k == "reynolds") c.reynolds = std::stod(v);
      else if(k == "lid_velocity") c.lid_velocity = std::stod(v);
      else if(k == "cfl_limit") c.cfl_limit = std::stod(v);
      else if(k == "max_steps") c.max_steps = std::stoi(v);
      else if(k == "min_steps") c.min_steps = std::stoi(v);
      else if(k == "steady_tolerance") c.steady_tolerance = std::stod(v);
      else if(k == "poisson_max_iterations") c.poisson_max_iterations = std::stoi(v);
      else if(k == "poisson_tolerance") c.poisson_tolerance = std::stod(v);
      else if(k == "validate_reference") c.validate_reference = parse_bool(v) ? 1 : 0;
      else throw std::runtime_error("unsupported cavity config key: " + k);
    });
    validate_cavity(c);
    *config = c;
  });
}

of_status of_cavity_config_describe(const of_cavity_config* config, char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    need(config, "config");
    const std::string s = cavity_describe(*config);
    if(buf) copy_text(buf, cap, s);
    if(len) *len = s.size();
  });
}

of_status of_cavity_case(const of_cavity_config* config, of_grid* grid, of_bc* bc, double* viscosity,
                         double* dt) {
  return guarded([&] {
    need(config, "config");
    if(grid) *grid = cavity_grid(*config);
    if(bc) *bc = cavity_bc(*config);
    if(viscosity) *viscosity = cavity_viscosity(*config);
    if(dt) *dt = cavity_dt(*config);
  });
}

of_status of_cavity_create(const of_cavity_config* config, int device, of_ctx** out) {
  return guarded([&] {
    need(config, "config");
    need(out, "output context pointer");
    *out = nullptr;
    validate_cavity(*config);
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    const of_grid g = cavity_grid(*config);
    const of_bc bc = cavity_bc(*config);
    of_ctx* ctx = nullptr;
    check(of_create(&g, &bc, device, &ctx));
    const of_status s = of_rest_init(ctx, cavity_viscosity(*config), cavity_dt(*config));
    if(s != OF_OK) {
      const std::string msg = of_last_error();
      of_destroy(ctx);
      throw Failure(s, msg);
    }
    *out = ctx;
  });
}

of_status of_cavity_run_steps(of_ctx* ctx, const of_cavity_config* config, int steps,
                              of_step_metrics* metrics) {
  return guarded([&] {
    need(config, "config");
    validate_cavity(*config);
    if(steps < 0) throw std::invalid_argument("run_lid_driven_cavity_steps expects a non-negative step count");
    require_cavity_state(ctx, *config);
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    const of_step_params p = cavity_params(*config);
    check(of_run_steps(ctx, &p, steps, metrics));
  });
}

of_status of_cavity_run_to_steady(of_ctx* ctx, const of_cavity_config* config, of_step_metrics* metrics) {
  return guarded([&] {
    need(config, "config");
    require_cavity_state(ctx, *config);
    require_step_scheme(config->advection_scheme, config->advection_limiter);
    const of_step_params p = cavity_params(*config);
    of_step_metrics m = ctx_metrics(ctx);
    while(m.step < config->max_steps) {
      check(of_run_steps(ctx, &p, 1, &m));
      if(steady(*config, m)) break;
    }
    if(metrics) *metrics = m;
  });
}

of_status of_cavity_centerlines(of_ctx* ctx, double* u_coordinate, double* u_value, double* v_coordinate,
                                double* v_value) {
  return guarded([&] {
    Profile pu, pv;
    centerlines(ctx, pu, pv);
    if(u_coordinate) std::copy(pu.x.begin(), pu.x.end(), u_coordinate);
    if(u_value) std::copy(pu.v.begin(), pu.v.end(), u_value);
    if(v_coordinate) std::copy(pv.x.begin(), pv.x.end(), v_coordinate);
    if(v_value) std::copy(pv.v.begin(), pv.v.end(), v_value);
  });
}

of_status of_cavity_finalize(of_ctx* ctx, const of_cavity_config* config, of_cavity_result* result) {
  return guarded([&] {
    need(config, "config");
    need(result, "result");
    require_cavity_state(ctx, *config);
    of_cavity_result r{};
    r.final_step = ctx_metrics(ctx);
    Profile pu, pv;
    centerlines(ctx, pu, pv);
    // compute_centerline_extrema (solver/lid_driven_cavity.cpp:133-154):
    // interior samples only.
    if(pu.v.size() < 3 || pv.v.size() < 3)
      throw std::invalid_argument("centerline extrema require at least three samples per profile");
    const auto u = std::minmax_element(pu.v.begin() + 1, pu.v.end() - 1);
    const auto v = std::minmax_element(pv.v.begin() + 1, pv.v.end() - 1);
    r.u_vertical_min = *u.first;
    r.u_vertical_max = *u.second;
    r.v_horizontal_min = *v.first;
    r.v_horizontal_max = *v.second;
    if(config->validate_reference && std::abs(config->reynolds - 100.0) < 1.0e-12) {
      copy_text(r.reference_dataset, sizeof(r.reference_dataset), kEnvelopeDataset);
      r.divergence_l2 = r.final_step.divergence_l2;
      bool pass = r.final_step.divergence_l2 <= 1.0e-10;
      double worst = 0.0;
      for(int q = 0; q < 4; ++q) {
        const EnvelopePoint& e = kEnvelope[q];
        of_cavity_point& out = r.points[q];
        copy_text(out.label, sizeof(out.label), e.label);
        out.line = e.line;
        out.coordinate = e.coordinate;
        out.reference_value = e.value;
        out.reference_lower_bound = e.lower;
        out.reference_upper_bound = e.upper;
        out.sample_value = profile_at(e.line == OF_U_VERTICAL ? pu : pv, e.coordinate);
        out.relative_error = envelope_miss(out.sample_value, e.lower, e.upper);
        worst = std::max(worst, out.relative_error);
        pass = pass && out.relative_error <= 0.02;
      }
      r.max_relative_error = worst;
      r.pass = pass ? 1 : 0;
    }
    *result = r;
  });
}

of_status of_cavity_run(of_ctx* ctx, const of_cavity_config* config, of_cavity_result* result) {
  return guarded([&] {
    need(config, "config");
    need(result, "result");
    require_cavity_state(ctx, *config);
    check(of_rest_init(ctx, cavity_viscosity(*config), cavity_dt(*config)));
    const auto t0 = Clock::now();
    check(of_cavity_run_to_steady(ctx, config, nullptr));
    const double elapsed = seconds_since(t0);
    check(of_cavity_finalize(ctx, config, result));
    result->elapsed_seconds = elapsed;
  });
}

// ---- checkpoint -------------------------------------------------------------

uint64_t of_fnv1a64(const void* data, size_t size) {
  return fnv_update(kFnvOffset, static_cast<const uint8_t*>(data), data ? size : 0);
}

uint64_t of_build_hash(const char* project_name, const char* project_version, const char* compiler_id,
                       const char* compiler_version, const char* build_profile, int fast_math_enabled) {
  const auto str = [](const char* s) { return std::string(s ? s : ""); };
  return fnv_text(str(project_name) + "|" + str(project_version) + "|" + str(compiler_id) + "|" +
                  str(compiler_version) + "|" + str(build_profile) + "|" +
                  (fast_math_enabled ? "fast-math" : "strict"));
}

uint64_t of_library_build_hash(void) { return library_build_hash(); }

of_status of_cavity_checkpoint_write(of_ctx* ctx, const char* path, const of_cavity_config* config,
                                     uint64_t build_hash) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    if(!same_grid(ctx_grid(ctx), cavity_grid(*config)))
      throw std::invalid_argument("checkpoint state grid does not match the cavity config");
    const HostState s = download_state(ctx);
    write_checkpoint(path, resolve_hash(build_hash), fnv_text(cavity_describe(*config)), "CONF",
                     cavity_config_bytes(*config), s, false);
  });
}

of_status of_cavity_checkpoint_load(of_ctx* ctx, const char* path, const of_cavity_config* config,
                                    uint64_t build_hash, of_checkpoint_meta* meta) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    if(!same_grid(ctx_grid(ctx), cavity_grid(*config)))
      throw std::invalid_argument("lid-driven cavity state grid does not match the config");
    of_checkpoint_meta m{};
    HostState s = load_checkpoint(path, cavity_expect(*config, resolve_hash(build_hash)), m);
    s.metrics.max_divergence_l2 = 0.0;
    upload_state(ctx, s);
    if(meta) *meta = m;
  });
}

of_status of_cavity_checkpoint_write_host(const char* path, const of_cavity_config* config,
                                          uint64_t build_hash, const double* u, const double* v,
                                          const double* w, const double* adv_u, const double* adv_v,
                                          const double* adv_w, const double* p_total,
                                          int has_previous_advection, const of_step_metrics* metrics) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    const double* f[7] = {u, v, w, adv_u, adv_v, adv_w, p_total};
    const HostState s = host_state(cavity_grid(*config), f, has_previous_advection, metrics);
    write_checkpoint(path, resolve_hash(build_hash), fnv_text(cavity_describe(*config)), "CONF",
                     cavity_config_bytes(*config), s, false);
  });
}

of_status of_cavity_checkpoint_load_host(const char* path, const of_cavity_config* config, uint64_t build_hash,
                                         double* u, double* v, double* w, double* adv_u, double* adv_v,
                                         double* adv_w, double* p_total, int* has_previous_advection,
                                         of_step_metrics* metrics, of_checkpoint_meta* meta) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    of_checkpoint_meta m{};
    const HostState s = load_checkpoint(path, cavity_expect(*config, resolve_hash(build_hash)), m);
    double* out[7] = {u, v, w, adv_u, adv_v, adv_w, p_total};
    for(int f = 0; f < 7; ++f)
      if(out[f]) std::copy(s.f[f].begin(), s.f[f].end(), out[f]);
    if(has_previous_advection) *has_previous_advection = s.has_prev;
    if(metrics) {
      *metrics = s.metrics;
      metrics->max_divergence_l2 = 0.0;
    }
    if(meta) *meta = m;
  });
}

of_status of_tg_checkpoint_write(of_ctx* ctx, const char* path, const of_tg_config* config,
                                 uint64_t build_hash) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    if(!same_grid(ctx_grid(ctx), tg_grid(*config)))
      throw std::invalid_argument("checkpoint state grid does not match the Taylor-Green config");
    const HostState s = download_state(ctx);
    write_checkpoint(path, resolve_hash(build_hash), fnv_text(tg_describe(*config)), "TGCF",
                     tg_config_bytes(*config), s, true);
  });
}

of_status of_tg_checkpoint_load(of_ctx* ctx, const char* path, const of_tg_config* config,
                                uint64_t build_hash, of_checkpoint_meta* meta) {
  return guarded([&] {
    need(path, "path");
    need(config, "config");
    require_tg_state(ctx, *config);
    of_checkpoint_meta m{};
    const HostState s = load_checkpoint(path, tg_expect(*config, resolve_hash(build_hash)), m);
    upload_state(ctx, s);
    if(meta) *meta = m;
  });
}

// ---- VTK --------------------------------------------------------------------

of_status of_write_vtk(of_ctx* ctx, const char* path) {
  return guarded([&] {
    need(path, "path");
    const HostState s = download_state(ctx);
    const of_grid& g = s.grid;
    std::unique_ptr<std::FILE, int (*)(std::FILE*)> file(std::fopen(path, "w"), &std::fclose);
    if(!file) throw std::runtime_error(std::string("unable to open VTK file for writing: ") + path);
    std::FILE* f = file.get();
    const auto idx = [](const std::array<int, 3>& e, int i, int j, int k) {
      return static_cast<size_t>(i) + static_cast<size_t>(e[0]) * (j + static_cast<size_t>(e[1]) * k);
    };
    const auto eu = storage(g, 0), ev = storage(g, 1), ew = storage(g, 2), ep = storage(g, 6);
    std::fprintf(f, "# vtk DataFile Version 3.0\nsolver checkpoint state\nASCII\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(f, "DIMENSIONS %d %d %d\nORIGIN ", g.nx, g.ny, g.nz);
    put_number(f, 0.5 * g.dx);
    std::fputc(' ', f);
    put_number(f, 0.5 * g.dy);
    std::fputc(' ', f);
    put_number(f, 0.5 * g.dz);
    std::fprintf(f, "\nSPACING ");
    put_number(f, g.dx);
    std::fputc(' ', f);
    put_number(f, g.dy);
    std::fputc(' ', f);
    put_number(f, g.dz);
    std::fprintf(f, "\nPOINT_DATA %zu\nVECTORS velocity double\n",
                 static_cast<size_t>(g.nx) * g.ny * g.nz);
    for(int k = 1; k <= g.nz; ++k)
      for(int j = 1; j <= g.ny; ++j)
        for(int i = 1; i <= g.nx; ++i) {
          put_number(f, 0.5 * (s.f[0][idx(eu, i, j, k)] + s.f[0][idx(eu, i + 1, j, k)]));
          std::fputc(' ', f);
          put_number(f, 0.5 * (s.f[1][idx(ev, i, j, k)] + s.f[1][idx(ev, i, j + 1, k)]));
          std::fputc(' ', f);
          put_number(f, 0.5 * (s.f[2][idx(ew, i, j, k)] + s.f[2][idx(ew, i, j, k + 1)]));
          std::fputc('\n', f);
        }
    std::fprintf(f, "SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    for(int k = 1; k <= g.nz; ++k)
      for(int j = 1; j <= g.ny; ++j)
        for(int i = 1; i <= g.nx; ++i) {
          put_number(f, s.f[6][idx(ep, i, j, k)]);
          std::fputc('\n', f);
        }
    if(std::ferror(f)) throw std::runtime_error(std::string("failed while writing VTK file: ") + path);
  });
}

}  // extern "C"

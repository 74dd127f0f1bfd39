// gs_plugins.cpp -- the registered systems of the front end.
//
// Dynamics_mart, Dynamics_precipitate and Dynamics_stress read the same
// `set` variables and fields as the reference's plugins
// (src/dynamics_mart.cu:14-173, src/dynamics_precipitate.cu:17-110,
// src/dynamics_stress.cu:19-113) and run the step through the C ABI
// (include/gs_capi.h).  `set model baseline` selects the project's
// discretisation with the extra keys landau / kappa / mobility / noise /
// appliedstress; the default is the reference's formulas.  Dynamics_pow is
// the reference's host-only demo (src/dynamics_pow.cu:18-47); Dynamics_cores
// makes the nuclei that start the precipitate chain.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/gs_capi.h"
#include "gs_driver.h"

namespace gsfe {

namespace {

std::string capi_error() {
  char buf[512];
  gs_last_error(buf, sizeof(buf));
  return buf;
}

// shared parameter parsing of the three physics plugins
struct PhysicsBase : Dynamics {
  gs_sim* sim = nullptr;
  gs_params p{};
  int V = 0;
  bool have_stats = false;
  gs_stats pre{};
  bool report_next = false;

  ~PhysicsBase() override {
    if (sim) gs_sim_destroy(sim);
  }

  std::string var(const std::string& k) { return (*Vars)[k]; }

  void grid() {
    std::string s = var("gridsize");
    if (!s.empty()) s >> nx >> ny >> nz >> dx >> dy >> dz;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.dx = dx;
    p.dy = dy;
    p.dz = dz;
  }

  int mode_from_vars() {
    std::string m;
    (void)(var("model") >>= m);
    return m == "baseline" ? GS_MODE_BASELINE : GS_MODE_REFCOMPAT;
  }

  void precision() {
    std::string s;
    (void)(var("precision") >>= s);
    if (s == "fp64") p.dtype = GS_DTYPE_F64;
  }

  int variants(const char* what) {
    Field* vt = Datas->find("varianttensor");
    if (!vt || vt->empty()) {
      log() << "Error: variants' strain tensor does not set while initialize dynamics\n";
      return kErr;
    }
    V = vt->dims[0];  // "3 V 3 3": the first extent counts the variants
    if (V < 1 || V > GS_MAX_V || vt->n() < (size_t)V * 9) {
      log() << "Error: varianttensor of " << what << " must be V x 3 x 3 with V <= " << GS_MAX_V << "\n";
      return kErr;
    }
    p.nvariants = V;
    for (int v = 0; v < V; ++v)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p.eigenstrain[v][i][j] = vt->v[(v * 3 + i) * 3 + j];
    return kNormal;
  }

  // a `modulus` field (3x3x3x3) replaces the default C_ijkl
  void modulus_field() {
    Field* m = Datas->find("modulus");
    if (m && m->n() == 81)
      for (int i = 0; i < 81; ++i) (&p.cijkl[0][0][0][0])[i] = m->v[i];
  }

  int create() {
    if (gs_sim_create(&p, &sim) != GS_OK) {
      log() << "Error: " << capi_error() << "\n";
      return kErr;
    }
    return kNormal;
  }

  // upload a field from the store, or create it with `fill`
  int field_in(const char* name, std::vector<int> dims, float fill, bool upload_if_present = true) {
    Field& f = (*Datas)[name];
    size_t n = 1;
    for (int d : dims) n *= (size_t)d;
    if (!f.empty() && f.n() == n) {
      if (upload_if_present && gs_sim_set_field(sim, name, f.v.data(), n, GS_DTYPE_F32) != GS_OK) {
        log() << "Error: " << capi_error() << "\n";
        return kErr;
      }
      return kNormal;
    }
    if (!f.empty()) {
      log() << "Error: field " << name << " has " << f.n() << " values, the grid needs " << n << "\n";
      return kErr;
    }
    f.init(dims, fill);
    return kNormal;
  }

  // the asynchronous dump job of a device field of extents `dims`
  Dynamics::DumpJob async_dump(const char* name, std::vector<int> dims) {
    int ticket = 0;
    if (gs_sim_copy_field_async(sim, name, nullptr, nullptr, &ticket) != GS_OK) return {};
    gs_sim* h = sim;
    return [h, ticket, dims](Field& f) -> std::string {
      f.init(dims);
      if (gs_sim_copy_field_wait(h, ticket, f.v.data(), f.n(), GS_DTYPE_F32) != GS_OK) return capi_error();
      return std::string();
    };
  }

  int sync(const char* name, std::vector<int> dims) {
    Field& f = (*Datas)[name];
    size_t n = 1;
    for (int d : dims) n *= (size_t)d;
    if (f.n() != n) f.init(dims);
    if (gs_sim_get_field(sim, name, f.v.data(), n, GS_DTYPE_F32) != GS_OK) {
      log() << "Error: " << capi_error() << "\n";
      return kErr;
    }
    return kNormal;
  }

  // statistics of the current state
  gs_stats now() {
    gs_stats s{};
    gs_sim_stats(sim, &s, nullptr);
    return s;
  }

  int step() {
    have_stats = false;
    if (report_next) {
      pre = now();  // force means of the state the step starts from
      have_stats = true;
    }
    if (gs_sim_step(sim, 1, nullptr) != GS_OK) {
      log() << "Error: " << capi_error() << "\n";
      return kErr;
    }
    return kNormal;
  }

  void WillReport(bool r) override { report_next = r; }

  // keys common to the physics plugins (FP64 device statistics)
  bool common_key(const std::string& k, std::string& out) {
    const gs_stats s = now();
    if (k == "mass") out = to_string6(s.mass);
    else if (k == "e_el") out = to_string6(s.e_el);
    else if (k == "e_chem") out = to_string6(s.e_chem);
    else if (k == "e_grad") out = to_string6(s.e_grad);
    else if (k == "e_appl") out = to_string6(s.e_appl);
    else if (k == "e_tot") out = to_string6(s.e_tot);
    else if (k == "c_mean") out = to_string6(s.c_mean);
    else if (k.rfind("vf", 0) == 0 && k.size() > 2) out = to_string6(s.vf[std::atoi(k.c_str() + 2) % GS_MAX_V]);
    else if (k.rfind("eta2_", 0) == 0) out = to_string6(s.eta2[std::atoi(k.c_str() + 5) % GS_MAX_V]);
    else return false;
    return true;
  }
};

class Mart : public PhysicsBase {
 public:
  float Temperature = 0;

  int Initialize() override {
    gs_params_default(&p, GS_MODEL_MART, mode_from_vars());
    grid();
    precision();
    std::string s;
    float f;
    if (p.mode == GS_MODE_REFCOMPAT) {
      f = (float)p.dt; (void)(var("deltatime") >>= f); p.dt = f;
      f = (float)p.transition_temperature; (void)(var("transitiontemperature") >>= f); p.transition_temperature = f;
      f = (float)p.weight_gradient; (void)(var("weightgradient") >>= f); p.weight_gradient = f;
      f = (float)p.weight_chemical; (void)(var("weightchemical") >>= f); p.weight_chemical = f;
      f = (float)p.weight_elastic; (void)(var("weightelastic") >>= f); p.weight_elastic = f;
      f = (float)p.weight_dislocation; (void)(var("weightdislocation") >>= f); p.weight_dislocation = f;
      f = (float)p.noise_amp; (void)(var("weightnoise") >>= f); p.noise_amp = f;
      s = var("coefficient");
      if (!s.empty()) {
        float a1 = 0, a2 = (float)p.lpc[2], a3 = (float)p.lpc[3];
        s >> a1 >> a2 >> a3;
        p.lpc[2] = a2;
        p.lpc[3] = a3;
      }
    } else {
      (void)(var("deltatime") >>= p.dt);
      s = var("landau");
      if (!s.empty()) s >> p.landau[0] >> p.landau[1] >> p.landau[2] >> p.landau[3];
      (void)(var("kappa") >>= p.kappa);
      (void)(var("mobility") >>= p.mobility);
      (void)(var("weightelastic") >>= p.weight_elastic);
      (void)(var("weightdislocation") >>= p.weight_dislocation);
      s = var("noise");
      if (!s.empty()) s >> p.noise_amp >> p.seed;
      s = var("appliedstress");  // xx yy zz yz xz xy
      if (!s.empty()) {
        double a[6] = {0, 0, 0, 0, 0, 0};
        s >> a[0] >> a[1] >> a[2] >> a[3] >> a[4] >> a[5];
        const int I[6] = {0, 1, 2, 1, 0, 0}, J[6] = {0, 1, 2, 2, 2, 1};
        memset(p.applied_stress, 0, sizeof(p.applied_stress));
        for (int k = 0; k < 6; ++k) p.applied_stress[I[k]][J[k]] = p.applied_stress[J[k]][I[k]] = a[k];
      }
    }
    s = var("seed");
    if (!s.empty()) s >> p.seed;
    if (variants("mart") != kNormal) return kErr;
    modulus_field();
    Temperature = (float)p.transition_temperature;
    p.temperature = Temperature;
    if (create() != kNormal) return kErr;
    if (field_in("eta", {V, nx, ny, nz}, 0.0f) != kNormal) return kErr;
    if (Field* d = Datas->find("defect"); d && !d->empty())
      if (gs_sim_set_field(sim, "defect", d->v.data(), d->n(), GS_DTYPE_F32) != GS_OK) {
        log() << "Error: " << capi_error() << "\n";
        return kErr;
      }
    if (Field* d = Datas->find("dislocationstress"); d && !d->empty())
      if (gs_sim_set_field(sim, "dislocationstress", d->v.data(), d->n(), GS_DTYPE_F32) != GS_OK) {
        log() << "Error: " << capi_error() << "\n";
        return kErr;
      }
    return kNormal;
  }

  int Calculate() override {
    (void)(var("temperature") >>= Temperature);
    gs_sim_set_scalar(sim, "temperature", Temperature);
    return step();
  }

  int RunFunc(std::string) override { return kNormal; }

  // `set fix temperature T0 T1`: the temperature of step i is
  // T0 + (i/n)(T1 - T0), stored as text (src/dynamics_mart.cu:421-441)
  int Fix(float progress) override {
    std::string s = var("fix");
    do {
      const std::string mode = take_word(s);
      if (mode == "temperature") {
        float st = 0, et = 0;
        s >> st >> et;
        (*Vars)["temperature"] <<= (st + progress * (et - st));
      } else if (mode == "pressure") {
      } else {
        log() << "Error: fix style " << mode << " does not find!\n";
      }
    } while (!s.empty());
    return kNormal;
  }

  std::string Get(std::string key) override {
    const std::string k = take_word(key);
    if (k == "temperature") return to_string6(Temperature);
    const gs_stats& f = have_stats ? pre : (pre = now());
    if (k == "eta") return to_string6(now().eta_mean);
    if (k == "gradient") return to_string6(f.gradient_mean);
    if (k == "chemical") return to_string6(f.chemical_mean);
    if (k == "elastic") return to_string6(f.elastic_mean);
    if (k == "dislocation") return to_string6(f.dislocation_mean);
    std::string out;
    if (common_key(k, out)) return out;
    return "nan";
  }

  int SyncToHost(const std::string& name) override {
    if (name == "eta") return sync("eta", {V, nx, ny, nz});
    return kNormal;
  }
  DumpJob DumpAsync(const std::string& name) override {
    if (name == "eta") return async_dump("eta", {V, nx, ny, nz});
    return {};
  }
};

class Precipitate : public PhysicsBase {
 public:
  float Temperature = 0;

  int Initialize() override {
    gs_params_default(&p, GS_MODEL_PRECIPITATE, mode_from_vars());
    grid();
    precision();
    std::string s;
    s = var("deltatime");
    if (!s.empty()) s >> p.dt;
    s = var("coefficient");
    if (!s.empty()) s >> p.coef[1] >> p.coef[2] >> p.coef[3] >> p.coef[4] >> p.coef[5] >> p.coef[6] >> p.coef[7];
    (void)(var("arfi") >>= p.kappa_eta);
    (void)(var("beta") >>= p.kappa_c);
    (void)(var("meta") >>= p.mobility_c);
    (void)(var("lpp") >>= p.mobility_eta);
    (void)(var("xi") >>= p.xi);
    s = var("concentration");
    if (!s.empty()) s >> p.c1 >> p.c2;
    (void)(var("weightnoise") >>= p.noise_amp);
    s = var("modulus");  // C00 C01 C33 (src/dynamics_precipitate.cu:55-65)
    if (!s.empty()) {
      double c00 = 3.5, c01 = 1.5, c33 = 1.0;
      s >> c00 >> c01 >> c33;
      memset(p.cijkl, 0, sizeof(p.cijkl));
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p.cijkl[i][i][j][j] = c01;
      for (int i = 0; i < 3; ++i) p.cijkl[i][i][i][i] = c00;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          if (i != j) p.cijkl[i][j][i][j] = p.cijkl[i][j][j][i] = c33;
    }
    if (p.mode == GS_MODE_BASELINE) {
      (void)(var("misfit") >>= p.misfit_c);
      s = var("noise");
      if (!s.empty()) s >> p.noise_amp >> p.seed;
    }
    s = var("seed");
    if (!s.empty()) s >> p.seed;
    if (variants("precipitate") != kNormal) return kErr;
    if (create() != kNormal) return kErr;
    const float c0 = (float)(p.c1 + (p.c2 - p.c1) / 3.0);
    if (field_in("concentration", {nx, ny, nz}, c0) != kNormal) return kErr;
    if (field_in("eta", {V, nx, ny, nz}, 0.0f) != kNormal) return kErr;
    return kNormal;
  }

  int Calculate() override {
    (void)(var("temperature") >>= Temperature);
    return step();
  }
  int RunFunc(std::string) override { return kNormal; }
  int Fix(float progress) override {
    std::string s = var("fix");
    while (!s.empty()) {
      const std::string mode = take_word(s);
      if (mode == "temperature") {
        float st = 0, et = 0;
        s >> st >> et;
        (*Vars)["temperature"] <<= (st + progress * (et - st));
      } else if (mode == "pressure") {
      } else {
        log() << "Error: fix style " << mode << " does not find!\n";
      }
    }
    return kNormal;
  }
  std::string Get(std::string key) override {
    const std::string k = take_word(key);
    if (k == "temperature") return to_string6(Temperature);
    if (k == "eta_average") return to_string6(now().eta_mean);
    std::string out;
    if (common_key(k, out)) return out;
    return "nan";
  }
  int SyncToHost(const std::string& name) override {
    if (name == "eta") return sync("eta", {V, nx, ny, nz});
    if (name == "concentration") return sync("concentration", {nx, ny, nz});
    return kNormal;
  }
  DumpJob DumpAsync(const std::string& name) override {
    if (name == "eta") return async_dump("eta", {V, nx, ny, nz});
    if (name == "concentration") return async_dump("concentration", {nx, ny, nz});
    return {};
  }
};

class Stress : public PhysicsBase {
 public:
  int Initialize() override {
    gs_params_default(&p, GS_MODEL_STRESS, mode_from_vars());
    grid();
    precision();
    (void)(var("xi") >>= p.xi);
    if (variants("stress") != kNormal) return kErr;
    modulus_field();
    if (create() != kNormal) return kErr;
    if (field_in("eta", {V, nx, ny, nz}, 0.0f) != kNormal) return kErr;
    (*Datas)["stress"].init({6, nx, ny, nz});
    (*Datas)["defect"].init({nx, ny, nz});
    return kNormal;
  }
  int Calculate() override { return step(); }
  int RunFunc(std::string) override { return kNormal; }
  int Fix(float) override { return kNormal; }
  std::string Get(std::string) override { return "nan"; }
  int SyncToHost(const std::string& name) override {
    if (name == "stress") return sync("stress", {6, nx, ny, nz});
    if (name == "defect") return sync("defect", {nx, ny, nz});
    return kNormal;
  }
  DumpJob DumpAsync(const std::string& name) override {
    if (name == "stress") return async_dump("stress", {6, nx, ny, nz});
    if (name == "defect") return async_dump("defect", {nx, ny, nz});
    return {};
  }
};

// the reference's demo system: `matrix` *= x every step
class Pow : public Dynamics {
 public:
  float x = 1.0f;
  Field* matrix = nullptr;
  int Initialize() override {
    (void)((*Vars)["x"] >>= x);
    matrix = &(*Datas)["matrix"];
    return kNormal;
  }
  int Calculate() override {
    for (float& v : matrix->v) v = v * x;
    return kNormal;
  }
  int RunFunc(std::string) override { return kUnknown; }
  int Fix(float) override { return kNormal; }
  std::string Get(std::string key) override {
    if (key == "x") return to_string6(x);
    if (key == "sum_of_matrix") return to_string6(matrix->sum());
    return "nan";
  }
};

// Dynamics_cores (src/dynamics_cores.cu:14-186): nuclei for the precipitate
// chain.  The placement makes the reference's draws from the C library's
// random() in the reference's order (random: a centre, redrawn while it lies
// in an earlier nucleus, then the variant; regular: one draw, then variant
// cn % V); the painting of the grid runs on the device (gs_cores_paint).
// regular2d / regular3d take the variant as random() % V: the reference's
// floor(random() * VariantN) overflows int and indexes eta out of range.
class Cores : public Dynamics {
 public:
  int V = 4, ncores = 5;
  float radius = 5.0f, c1 = 0.2f, c2 = 0.44f;
  std::string method = "random";
  Field* eta = nullptr;
  Field* conc = nullptr;

  int Initialize() override {
    nx = ny = nz = 16;
    dx = dy = dz = 0.1f;
    std::string s = (*Vars)["gridsize"];
    if (!s.empty()) s >> nx >> ny >> nz >> dx >> dy >> dz;
    (void)((*Vars)["variantn"] >>= V);
    (void)((*Vars)["coresn"] >>= ncores);
    (void)((*Vars)["radius"] >>= radius);
    s = (*Vars)["concentration"];
    if (!s.empty()) s >> c1 >> c2;
    s = (*Vars)["method"];
    if (!s.empty()) method = take_word(s);
    eta = &(*Datas)["eta"];
    eta->init({V, nx, ny, nz}, 0.0f);
    conc = &(*Datas)["concentration"];
    conc->init({nx, ny, nz}, c1);
    return kNormal;
  }

  bool marked(const std::vector<int>& cen, int i, int j, int k) const {
    const double r = (double)radius, r2 = r * r;
    for (size_t q = 0; q + 2 < cen.size(); q += 3) {
      const double x = i - cen[q], y = j - cen[q + 1], z = k - cen[q + 2];
      auto in = [r2](double a, double b, double c) { return a * a + b * b + c * c <= r2; };
      if (in(x, y, z) || in(x + nx, y, z) || in(x - nx, y, z) || in(x, y + ny, z) || in(x, y - ny, z) ||
          in(x, y, z + nz) || in(x, y, z - nz))
        return true;
    }
    return false;
  }

  int Calculate() override {
    std::vector<int> cen, var;
    if (method == "random") {
      for (int cn = 0; cn < ncores; ++cn) {
        int ox = 0, oy = 0, oz = 0;
        for (int j = 0; j < 100000; ++j) {
          ox = (int)(random() % nx);
          oy = (int)(random() % ny);
          oz = (int)(random() % nz);
          if (!marked(cen, ox, oy, oz)) break;
        }
        cen.insert(cen.end(), {ox, oy, oz});
        var.push_back((int)(random() % V));
      }
    } else if (method == "regular") {
      for (int cn = 0; cn < ncores; ++cn) {
        (void)random();
        cen.insert(cen.end(), {nx / 2, ny / 2, nz / ncores / 2 + nx / ncores * cn});
        var.push_back(cn % V);
      }
    } else if (method == "regular2d") {
      for (int c1i = 0; c1i < ncores; ++c1i)
        for (int c2i = 0; c2i < ncores; ++c2i) {
          cen.insert(cen.end(), {nx / 2, ny / ncores / 2 + ny / ncores * c2i, nz / ncores / 2 + nx / ncores * c1i});
          var.push_back((int)(random() % V));
        }
    } else if (method == "regular3d") {
      for (int c1i = 0; c1i < ncores; ++c1i)
        for (int c2i = 0; c2i < ncores; ++c2i)
          for (int c3i = 0; c3i < ncores; ++c3i) {
            cen.insert(cen.end(), {nx / ncores / 2 + nx / ncores * c3i, ny / ncores / 2 + ny / ncores * c2i,
                                   nz / ncores / 2 + nx / ncores * c1i});
            var.push_back((int)(random() % V));
          }
    } else {
      return kNormal;  // the reference paints nothing for another method
    }
    if (gs_cores_paint(nx, ny, nz, V, (int)var.size(), cen.data(), var.data(), radius, c1, c2, eta->v.data(),
                       conc->v.data()) != GS_OK) {
      log() << "Error: " << capi_error() << "\n";
      return kErr;
    }
    return kNormal;
  }
  int RunFunc(std::string) override { return kNormal; }
  int Fix(float) override { return kNormal; }
  std::string Get(std::string) override { return "nan"; }
};

}  // namespace

std::unique_ptr<Dynamics> make_dynamics(const std::string& name) {
  if (name == "cores") return std::make_unique<Cores>();
  if (name == "mart") return std::make_unique<Mart>();
  if (name == "precipitate") return std::make_unique<Precipitate>();
  if (name == "stress") return std::make_unique<Stress>();
  if (name == "pow") return std::make_unique<Pow>();
  return nullptr;
}

}  // namespace gsfe

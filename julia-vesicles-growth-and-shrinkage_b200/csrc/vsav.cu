// C ABI of libvsav (declared in include/vsav.h).
#include "../../include/vsav.h"
#include "solver.cuh"

#include <cstring>
#include <string>

using namespace vsav;

struct vsav_handle {
  SolverBase* s = nullptr;
  int R = 1, V = 1, nd = 2;
  int device = 0;
  std::string err;
};

namespace {

thread_local std::string g_create_error;

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

int code_of(const std::string& m) { return (m.rfind("CUDA", 0) == 0) ? VSAV_E_CUDA : VSAV_E_INVALID; }

template <typename F>
int guard(vsav_handle* h, F&& f) {
  if (!h || !h->s) return VSAV_E_INVALID;
  try {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e));
    return f();
  } catch (const std::exception& e) {
    h->err = e.what();
    return code_of(h->err);
  }
}

int check_status(vsav_handle* h, vsav_status* out) {
  StepStatus s = h->s->status();
  if (out) {
    out->err_flags = s.err_flags;
    out->psi_systems = s.psi_systems;
    out->psi_max_iters = s.psi_max_iters;
    out->psi_not_converged = s.psi_not_converged;
  }
  if (s.err_flags & 7) {
    h->err = "FATAL: W + C < 0 (flags " + std::to_string(s.err_flags) + ")";
    return VSAV_E_WC_NEGATIVE;
  }
  if (s.err_flags) {                // 8: a Krylov loop hit its bound; 16: a tile-copy wait timed out
    h->err = "CUDA error: device-side bound exceeded (flags " + std::to_string(s.err_flags) + ")";
    return VSAV_E_CUDA;
  }
  return s.psi_not_converged ? VSAV_W_NOT_CONVERGED : VSAV_OK;
}

int check_finite(vsav_handle* h) {
  std::vector<double> q(4 * h->R);
  h->s->get_scalars(0, q.data());
  for (double x : q)
    if (!std::isfinite(x)) { h->err = "non-finite SAV scalar (Q/R1/R2/R3)"; return VSAV_E_NONFINITE; }
  return VSAV_OK;
}

}  // namespace

extern "C" {

const char* vsav_last_error(const vsav_handle* h) { return h ? h->err.c_str() : ""; }
const char* vsav_create_error(void) { return g_create_error.c_str(); }

void vsav_default_options(vsav_options* o, const vsav_config* cfg) {
  std::memset(o, 0, sizeof(*o));
  o->precision = VSAV_FP64;
  o->psi_form = VSAV_PSI_FULL;
  o->psi_precond = 0;
  o->psi_itmax = 20;
  o->psi_rtol = cfg ? cfg->tol : 1e-12;
  o->psi_atol = 1e-14;
  o->n_runs = 1;
  o->run_sizes = nullptr;
  o->device = 0;
  o->graph = 1;
  o->psi3d_variable = 0;
  o->psi_stop = 0;
  o->psi_check = 0;
}

int vsav_create(const vsav_config* cfg, const vsav_options* opt, vsav_handle** out) {
  if (!cfg || !out) return VSAV_E_INVALID;
  *out = nullptr;
  vsav_options o;
  if (opt) o = *opt; else vsav_default_options(&o, cfg);
  auto* h = new vsav_handle();
  h->device = o.device;
  try {
    if (cfg->ndim != 2 && cfg->ndim != 3) throw std::runtime_error("ndim must be 2 or 3");
    const int E = (o.precision == VSAV_FP32) ? 16 : 8;
    const int CH = (o.precision == VSAV_FP32) ? 4096 : 2048;
    auto ok = [&](int n, int lo, int hi) { return is_pow2(n) && n >= lo && n <= hi; };
    if (!ok(cfg->Nx, 32, 2 * CH)) throw std::runtime_error("Nx must be a power of two in [32, " + std::to_string(2 * CH) + "]");
    if (!ok(cfg->Ny, E, CH)) throw std::runtime_error("Ny must be a power of two in [" + std::to_string(E) + ", " + std::to_string(CH) + "]");
    if (cfg->ndim == 3 && !ok(cfg->Nz, E, CH)) throw std::runtime_error("Nz must be a power of two in [" + std::to_string(E) + ", " + std::to_string(CH) + "]");
    if (cfg->ndim == 2 && o.psi_form == VSAV_PSI_FULL && cfg->Nx > CH) throw std::runtime_error("Nx too large for the full-spectrum psi form");
    if (o.n_runs < 1) throw std::runtime_error("n_runs must be >= 1");
    if (o.psi_itmax < 0) throw std::runtime_error("psi_itmax must be >= 0");
    std::vector<int> rs(o.n_runs);
    int V = 0;
    for (int r = 0; r < o.n_runs; ++r) {
      rs[r] = o.run_sizes ? o.run_sizes[r] : cfg->N;
      if (rs[r] < 1) throw std::runtime_error("every run needs at least one vesicle field");
      V += rs[r];
    }
    if (cfg->ndim == 3 && V != o.n_runs) throw std::runtime_error("3D runs hold one vesicle field each (the coupling of Solvers_3d.jl:260-267 is defined for N == 1)");
    if (!cfg->psi_in_v || !cfg->psi_out_v) throw std::runtime_error("psi_in_v / psi_out_v are required");
    cudaError_t e = cudaSetDevice(o.device);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e));
    Dims d{cfg->ndim, cfg->Nx, cfg->Ny, cfg->ndim == 3 ? cfg->Nz : 1, V, o.n_runs, cfg->Lx, cfg->Ly, cfg->ndim == 3 ? cfg->Lz : 1.0};
    Phys p{};
    p.eps = cfg->epsilon; p.M_phi = cfg->M_phi; p.M0_psi = cfg->M0_psi; p.eta = cfg->eta;
    p.gamma_surf = cfg->gamma_surf; p.gamma_area = cfg->gamma_area; p.gamma_bend = cfg->gamma_bend;
    p.gamma_in = cfg->gamma_in; p.beta_in = cfg->beta_in; p.gamma_out = cfg->gamma_out; p.beta_out = cfg->beta_out;
    p.lamda = cfg->lamda; p.S1 = cfg->S1; p.S2 = cfg->S2; p.S3 = cfg->S3; p.S4 = cfg->S4;
    p.C1 = cfg->C1; p.C2 = cfg->C2; p.C3 = cfg->C3;
    p.cell = (cfg->Lx / cfg->Nx) * (cfg->Ly / cfg->Ny) * (cfg->ndim == 3 ? cfg->Lz / cfg->Nz : 1.0);
    p.conf_dt = cfg->dt;
    Options so;
    so.precision = o.precision; so.psi_form = o.psi_form; so.psi_precond = o.psi_precond;
    so.psi_itmax = o.psi_itmax; so.psi_rtol = o.psi_rtol; so.psi_atol = o.psi_atol;
    if (o.precision != VSAV_FP64 && o.precision != VSAV_FP32 && o.precision != VSAV_MIXED)
      throw std::runtime_error("precision must be VSAV_FP64, VSAV_FP32 or VSAV_MIXED");
    so.graph = o.graph ? 1 : 0;
    if (o.psi_stop != 0 && o.psi_stop != 1) throw std::runtime_error("psi_stop must be 0 or 1");
    so.psi_stop = o.psi_stop;
    so.psi_check = o.psi_check ? 1 : 0;
    so.psi3d_var = (cfg->ndim == 3 && o.psi3d_variable) ? 1 : 0;
    // mixed: the psi BiCGSTAB in FP32 inside FP64 refinement wherever there is one (2D, 3D variable
    // mobility); otherwise (3D constant mobility) every field stays FP64
    so.psi_mixed = (o.precision == VSAV_MIXED && (cfg->ndim == 2 || so.psi3d_var)) ? 1 : 0;
    if (so.psi3d_var) {
      if (o.psi_form != VSAV_PSI_FULL) throw std::runtime_error("the 3D variable-mobility psi solve uses the full-spectrum form");
      if (o.psi_precond != 0) throw std::runtime_error("the 3D variable-mobility psi solve uses the diagonal preconditioner (psi_precond 0)");
      if (cfg->Nx > CH) throw std::runtime_error("Nx too large for the full-spectrum psi form");
    }
    if (o.precision == VSAV_FP32)
      h->s = make_solver_f32(d, p, so, rs.data(), cfg->psi_in_v, cfg->psi_out_v);
    else
      h->s = make_solver_f64(d, p, so, rs.data(), cfg->psi_in_v, cfg->psi_out_v);
    h->R = o.n_runs; h->V = V; h->nd = cfg->ndim;
    std::vector<double> dt(o.n_runs, cfg->dt);
    h->s->set_dt(dt.data());
  } catch (const std::exception& ex) {
    g_create_error = ex.what();
    int code = code_of(g_create_error);
    delete h->s;
    delete h;
    return code;
  }
  *out = h;
  return VSAV_OK;
}

int vsav_destroy(vsav_handle* h) {
  if (!h) return VSAV_E_INVALID;
  cudaSetDevice(h->device);
  delete h->s;
  delete h;
  return VSAV_OK;
}

int vsav_set_field(vsav_handle* h, int32_t level, int32_t field, const double* data) {
  return guard(h, [&] {
    if ((level != 0 && level != 1) || field < 0 || field > VSAV_NU_HAT || !data) throw std::runtime_error("bad field/level");
    h->s->set_field(level, field, data, 0);
    return VSAV_OK;
  });
}
int vsav_get_field(vsav_handle* h, int32_t level, int32_t field, double* data) {
  return guard(h, [&] {
    if ((level != 0 && level != 1) || field < 0 || field > VSAV_NU_HAT || !data) throw std::runtime_error("bad field/level");
    h->s->get_field(level, field, data);
    return VSAV_OK;
  });
}
int vsav_export_f32(vsav_handle* h, int32_t level, int32_t what, float* data) {
  return guard(h, [&] {
    const bool ok = what == VSAV_EXPORT_PHI_SUM || what == VSAV_EXPORT_SPEED ||
                    (what >= VSAV_EXPORT_FIELD && what <= VSAV_EXPORT_FIELD + VSAV_NU_HAT && (what - VSAV_EXPORT_FIELD) % 2 == 0);
    if ((level != 0 && level != 1) || !ok || !data) throw std::runtime_error("bad export id/level");
    h->s->export_f32(level, what, data);
    return VSAV_OK;
  });
}
int vsav_set_scalars(vsav_handle* h, int32_t level, const double* q4) {
  return guard(h, [&] { if (!q4 || (level != 0 && level != 1)) throw std::runtime_error("bad args"); h->s->set_scalars(level, q4); return VSAV_OK; });
}
int vsav_get_scalars(vsav_handle* h, int32_t level, double* q4) {
  return guard(h, [&] { if (!q4 || (level != 0 && level != 1)) throw std::runtime_error("bad args"); h->s->get_scalars(level, q4); return VSAV_OK; });
}
int vsav_set_dt(vsav_handle* h, const double* dt) {
  return guard(h, [&] {
    if (!dt) throw std::runtime_error("bad args");
    for (int r = 0; r < h->R; ++r) if (!(dt[r] > 0)) throw std::runtime_error("dt must be > 0");
    h->s->set_dt(dt);
    return VSAV_OK;
  });
}
int vsav_get_dt(vsav_handle* h, double* dt) {
  return guard(h, [&] { if (!dt) throw std::runtime_error("dt is NULL"); h->s->get_dt(dt); return VSAV_OK; });
}
int vsav_set_A0(vsav_handle* h, const double* a0) {
  return guard(h, [&] { if (!a0) throw std::runtime_error("bad args"); h->s->set_A0(a0); return VSAV_OK; });
}
int vsav_get_A0(vsav_handle* h, double* a0) {
  return guard(h, [&] { if (!a0) throw std::runtime_error("bad args"); h->s->get_A0(a0); return VSAV_OK; });
}
int vsav_init_shapes2d(vsav_handle* h, const vsav_shape2d* shapes) {
  return guard(h, [&] {
    if (!shapes) throw std::runtime_error("shapes is NULL");
    static_assert(sizeof(vsav_shape2d) == sizeof(Shape2D), "shape struct layouts differ");
    std::vector<Shape2D> s(h->V);
    std::memcpy(s.data(), shapes, h->V * sizeof(Shape2D));
    h->s->init_shapes2d(s.data());
    return check_status(h, nullptr) < 0 ? VSAV_E_WC_NEGATIVE : VSAV_OK;
  });
}
int vsav_generate_initial_condition(vsav_handle* h, int32_t state_type, int32_t goal, const double* blob_u) {
  return guard(h, [&] {
    h->s->init_reference_shapes(state_type, goal, blob_u);
    return check_status(h, nullptr) < 0 ? VSAV_E_WC_NEGATIVE : VSAV_OK;
  });
}
int vsav_init_state(vsav_handle* h, int32_t hats_given) {
  return guard(h, [&] { h->s->init_state(hats_given); return check_status(h, nullptr) < 0 ? VSAV_E_WC_NEGATIVE : VSAV_OK; });
}
int vsav_step1(vsav_handle* h, int32_t n, vsav_status* st) {
  return guard(h, [&] { if (n < 1) throw std::runtime_error("n >= 1"); h->s->step1(n); h->s->sync(); return check_status(h, st); });
}
int vsav_step2(vsav_handle* h, int32_t n) {
  return guard(h, [&] { if (n < 1) throw std::runtime_error("n >= 1"); h->s->step2(n); h->s->sync(); return VSAV_OK; });
}
int vsav_step3(vsav_handle* h) { return guard(h, [&] { h->s->step3(); h->s->sync(); return VSAV_OK; }); }
int vsav_step4(vsav_handle* h, int32_t n) {
  return guard(h, [&] { if (n < 1) throw std::runtime_error("n >= 1"); h->s->step4(n); h->s->sync(); return VSAV_OK; });
}
int vsav_step5(vsav_handle* h, int32_t n) {
  return guard(h, [&] { if (n < 1) throw std::runtime_error("n >= 1"); h->s->step5(n); h->s->sync(); return VSAV_OK; });
}
int vsav_step6(vsav_handle* h) { return guard(h, [&] { h->s->step6(); h->s->sync(); return VSAV_OK; }); }
int vsav_step7(vsav_handle* h, int32_t n) {
  return guard(h, [&] { if (n < 1) throw std::runtime_error("n >= 1"); h->s->step7(n); h->s->sync(); return VSAV_OK; });
}
int vsav_update_state(vsav_handle* h) {
  return guard(h, [&] { h->s->update_state(); h->s->sync(); return check_finite(h); });
}
int vsav_run(vsav_handle* h, int32_t n0, int32_t nsteps, const double* dt, double* energy, double* area_ratio, vsav_status* st) {
  return guard(h, [&] {
    if (n0 < 1 || nsteps < 0) throw std::runtime_error("bad step range");
    int worst = VSAV_OK;
    std::vector<double> e(h->R), a(h->R);
    const bool mon = energy || area_ratio;
    // st reports the first step whose psi solve did not converge, else the last step
    vsav_status cur{}, first_bad{};
    bool bad = false;
    auto note = [&](int rc) {
      if (rc > 0 && !bad) { first_bad = cur; bad = true; }
      if (st) *st = bad ? first_bad : cur;
    };
    for (int k = 0; k < nsteps; ++k) {
      if (dt) h->s->set_dt(dt + (size_t)k * h->R);
      int n = n0 + k;
      // whole step from a CUDA graph (errors of the step are read after it)
      if (h->s->step_graph(n, mon ? e.data() : nullptr, mon ? a.data() : nullptr)) {
        int rc = check_status(h, &cur);
        note(rc);
        if (rc < 0) return rc;
        if (rc > 0) worst = rc;
        for (int r = 0; r < h->R; ++r) {
          if (energy) energy[(size_t)k * h->R + r] = e[r];
          if (area_ratio) area_ratio[(size_t)k * h->R + r] = a[r];
        }
        continue;
      }
      h->s->step1(n);
      int rc = check_status(h, &cur);
      note(rc);
      if (rc < 0) return rc;
      if (rc > 0) worst = rc;
      h->s->step2(n); h->s->step3(); h->s->step4(n); h->s->step5(n); h->s->step6(); h->s->step7(n);
      h->s->update_state();
      if (mon) {
        h->s->monitor(e.data(), a.data());
        for (int r = 0; r < h->R; ++r) {
          if (energy) energy[(size_t)k * h->R + r] = e[r];
          if (area_ratio) area_ratio[(size_t)k * h->R + r] = a[r];
        }
      }
    }
    h->s->sync();
    int rc = check_finite(h);
    return rc < 0 ? rc : worst;
  });
}
int vsav_monitor(vsav_handle* h, double* energy, double* area_ratio) {
  return guard(h, [&] { h->s->monitor(energy, area_ratio); return VSAV_OK; });
}
int vsav_get_work(vsav_handle* h, int32_t what, int32_t idx, double* out) {
  return guard(h, [&] {
    bool ok = out && ((what == 0 && idx >= 0 && idx < 16) || (what == 1 && idx >= 0 && idx < 8) ||
                      ((what == 2 || what == 3) && (idx == 0 || idx == 1)) || (what == 4 && idx >= 0 && idx < 4));
    if (!ok) throw std::runtime_error("bad work id");
    h->s->get_work(what, idx, out);
    return VSAV_OK;
  });
}
int vsav_get_scalar_work(vsav_handle* h, int32_t what, double* out) {
  return guard(h, [&] {
    if (!out || what < 0 || what > 6) throw std::runtime_error("bad scalar work id");
    h->s->get_scalar_work(what, out);
    return VSAV_OK;
  });
}
int vsav_time_run(vsav_handle* h, int32_t n0, int32_t nsteps, const double* dt, int32_t monitor, double* device_ms) {
  return guard(h, [&] {
    if (!device_ms) throw std::runtime_error("bad args");
    cudaEvent_t a, b;
    VSAV_CUDA(cudaEventCreate(&a));
    VSAV_CUDA(cudaEventCreate(&b));
    h->s->sync();
    VSAV_CUDA(cudaEventRecord(a, h->s->stream()));
    std::vector<double> e(monitor ? (size_t)nsteps * h->R : 0), ar(e.size());
    int rc = vsav_run(h, n0, nsteps, dt, monitor ? e.data() : nullptr, monitor ? ar.data() : nullptr, nullptr);
    VSAV_CUDA(cudaEventRecord(b, h->s->stream()));
    VSAV_CUDA(cudaEventSynchronize(b));
    float t = 0;
    VSAV_CUDA(cudaEventElapsedTime(&t, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *device_ms = t;
    return rc;
  });
}
int64_t vsav_launch_count(void) { return (int64_t)launch_counter().load(); }

int vsav_get_tuning(vsav_handle* h, char* buf, int64_t cap, int64_t* needed) {
  return guard(h, [&] {
    const std::string t = h->s->tuning();
    if (needed) *needed = (int64_t)t.size() + 1;
    if (buf) {
      if (cap < (int64_t)t.size() + 1) throw std::runtime_error("tuning buffer too small");
      memcpy(buf, t.c_str(), t.size() + 1);
    }
    return VSAV_OK;
  });
}

int vsav_profile(vsav_handle* h, int32_t enable) {
  return guard(h, [&] { h->s->profile(enable); return VSAV_OK; });
}
int vsav_profile_read(vsav_handle* h, int32_t kclass, double* out3) {
  return guard(h, [&] {
    if (!out3 || kclass < 0 || kclass >= KC_N) throw std::runtime_error("bad kernel class");
    h->s->profile_read(kclass, out3);
    return VSAV_OK;
  });
}

int vsav_transform(vsav_handle* h, int32_t kind, int32_t nf, const double* in, double* out) {
  return guard(h, [&] {
    bool ok = in && out && nf >= 1 && nf <= 3 * h->V && (kind == 0 || kind == 1 || (kind >= 11 && kind <= 15));
    if (!ok) throw std::runtime_error("bad transform arguments");
    if (kind == 13 && h->nd != 3) throw std::runtime_error("D1z needs a 3D handle");
    h->s->transform(kind, nf, in, out);
    return VSAV_OK;
  });
}

int vsav_set_psi_net(vsav_handle* h, const double* theta) {
  return guard(h, [&] {
    if (!theta) throw std::runtime_error("theta is NULL");
    if (h->nd != 2) throw std::runtime_error("the learned psi preconditioner is 2D only");
    std::vector<float> wb(NET_NPARAM);
    for (int k = 0; k < NET_NPARAM; ++k) wb[k] = (float)theta[k];
    for (int l = 0; l < NET_NL; ++l)
      for (int k = net_woff(l); k < net_woff(l) + net_wsize(l); ++k) wb[k] = bf16_round(wb[k]);
    std::vector<uint32_t> fr(NF_WORDS);
    std::vector<float> bias(NF_BIAS, 0.f);
    net_pack(wb.data(), fr.data(), bias.data());
    std::vector<uint16_t> img(NT_WBYTES / 2);
    net_pack_tc(wb.data(), img.data());
    h->s->set_psi_net(fr.data(), bias.data(), img.data());
    return VSAV_OK;
  });
}

int vsav_psi_harvest(vsav_handle* h, int32_t max_snapshots) {
  return guard(h, [&] { h->s->harvest(max_snapshots); return VSAV_OK; });
}

int vsav_psi_harvest_read(vsav_handle* h, float* out, int64_t capacity, int32_t* nsnap, int64_t* nfloats) {
  return guard(h, [&] {
    int ns = 0;
    long long need = h->s->harvest_read(out, capacity, &ns);
    if (nsnap) *nsnap = ns;
    if (nfloats) *nfloats = need;
    return VSAV_OK;
  });
}

}  // extern "C"

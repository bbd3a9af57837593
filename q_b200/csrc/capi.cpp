// capi.cpp -- host-side entry points of the C ABI (include/qb.h): systems,
// files and errors.  Batch entry points live in engine.cu.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "qsystem.hpp"

namespace qb {
thread_local std::string g_last_error;
void set_error(const std::string &m) { g_last_error = m; }

// Run f, mapping exceptions to status codes; never lets one cross the ABI.
template <class F>
int guarded(F &&f) {
  try {
    f();
    return QB_OK;
  } catch (const Error &e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_error("out of host memory");
    return QB_ERR_ARG;
  } catch (const std::exception &e) {
    set_error(e.what());
    return QB_ERR_ARG;
  } catch (...) {
    set_error("unknown error");
    return QB_ERR_ARG;
  }
}

const System *system_of(const qb_handle *h) { return &h->sys; }
}  // namespace qb

using qb::guarded;

extern "C" {

int qb_version(char *buf, size_t n) {
  if (!buf || n == 0) return QB_ERR_ARG;
  std::snprintf(buf, n, "qb 0.1.0 (sm_100a)");
  return QB_OK;
}

int qb_last_error(char *buf, size_t n) {
  if (!buf || n == 0) return QB_ERR_ARG;
  std::snprintf(buf, n, "%s", qb::g_last_error.c_str());
  return QB_OK;
}

int qb_open_override(const char *inp_path, const qb_options *opt, const double *lambdas, int n_lambda,
                     int seed, qb_handle **out) {
  if (!inp_path || !out) { qb::set_error("null argument"); return QB_ERR_ARG; }
  *out = nullptr;
  (void)opt;
  qb_handle *h = nullptr;
  int rc = guarded([&] {
    h = new qb_handle();
    qb::read_inp(inp_path, h->sys.in);
    if (n_lambda > 0) {
      if (n_lambda > QB_MAX_STATES) qb::fail(QB_ERR_ARG, "too many lambda values");
      h->sys.in.lambdas.assign(lambdas, lambdas + n_lambda);
    }
    if (seed >= 0) {
      h->sys.in.iseed = seed;
      if (seed > 0 && !h->sys.in.have_tmaxw) qb::fail(QB_ERR_ARG, "seed override needs initial_temperature in the input");
    }
    qb::prepare(h->sys);
  });
  if (rc != QB_OK) { delete h; return rc; }
  *out = h;
  return QB_OK;
}

int qb_open(const char *inp_path, const qb_options *opt, qb_handle **out) {
  return qb_open_override(inp_path, opt, nullptr, 0, -1, out);
}

int qb_get_view(const qb_handle *h, qb_sysview *out) {
  if (!h || !out) { qb::set_error("null argument"); return QB_ERR_ARG; }
  h->sys.fill_view(out);
  return QB_OK;
}

void qb_close(qb_handle *h) { delete h; }

int qb_write_re(const char *path, int natom, const double *x, const double *v, int nshell, const float *theta_corr) {
  if (!path || natom <= 0 || !x || !v) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded([&] { qb::write_restart(path, natom, x, v, nshell, theta_corr); });
}

int qb_write_re_box(const char *path, int natom, const double *x, const double *v, int nshell,
                    const float *theta_corr, const double *box6) {
  if (!path || natom <= 0 || !x || !v || !box6) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded([&] { qb::write_restart(path, natom, x, v, nshell, theta_corr, box6); });
}

int qb_append_en(const char *path, int nstates, const double *EQ) {
  if (!path || nstates < 0 || (nstates > 0 && !EQ)) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded([&] { qb::append_energy_frame(path, nstates, EQ, 0, nullptr, nullptr); });
}

int qb_append_en_offd(const char *path, int nstates, const double *EQ, int noffd, const int *ij, const double *hr) {
  if (!path || nstates < 0 || (nstates > 0 && !EQ) || noffd < 0 || (noffd > 0 && (!ij || !hr))) {
    qb::set_error("invalid argument");
    return QB_ERR_ARG;
  }
  return guarded([&] { qb::append_energy_frame(path, nstates, EQ, noffd, ij, hr); });
}

// Maxwell-Boltzmann velocities exactly as maxwell/gauss/randm draw them
// (md.f90:3787-3810, 1453-1469, 14408-14442), before initial shaking.
int qb_maxwell(int seed, double temperature, int natom, const double *mass, double *v_out) {
  if (natom < 0 || !mass || !v_out) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  const int m = 100000000, m1 = 10000, mult = 31415821;
  int irand = std::abs(seed) % m;
  double kT = (double)qb::kBoltz * temperature;
  for (int i = 0; i < natom; i++) {
    double sd = std::sqrt(kT / mass[i]);
    for (int k = 0; k < 3; k++) {
      double a = 0.0;
      for (int r = 0; r < 12; r++) {
        int irandh = irand / m1, irandl = irand % m1;
        irand = (((irandh * (mult % m1) + irandl * (mult / m1)) % m1) * m1 + irandl * (mult % m1));
        irand = (irand + 1) % m;
        float rv = (float)(irand / 10) * 10.0f / (float)m;
        if (rv <= 0.0f || rv > 1.0f) rv = 0.0f;
        a += (double)rv;
      }
      v_out[3 * i + k] = (a - 6.0) * sd + 0.0;
    }
  }
  return QB_OK;
}

}  // extern "C"

// agpu_ionz.cpp — host-side ADK one-level ionization tables.
//
// Restates set_ionization_coeff (src/ionization/ionz_data.f90:131-245,
// 770-804) and the one-level branch of set_field_ioniz_wfunction
// (src/ionization/ionize.f90:38-190).  The table is built once on the host in
// FP64 with the C library's exp/pow (as the reference does with its own
// runtime) and uploaded; the device only indexes it, so no device libm
// enters the ionization decision.
#include <cmath>
#include <cstring>
#include <vector>

#include "agpu_ionz.h"

namespace agpu {

namespace {
struct Adk {
  double v[8], v_norm[8], e_c[8], nstar[8], vfact[8], e_b[8], c_nstar[8];
  int l_fact[8];
};

bool adk_coeff(int an, Adk& a) {
  const double v_h = 13.5984, euler = 2.71828, pig = 3.141592653589793;
  std::memset(&a, 0, sizeof(a));
  for (int i = 0; i < 8; ++i) a.l_fact[i] = 1;
  switch (an) {
    case 1:  // H: 1s
      a.v[1] = 13.5984;
      break;
    case 2:  // He: 1s^2
      a.v[1] = 24.5874;
      a.v[2] = 54.41776;
      break;
    case 3:  // Li: [He] 2s
      a.v[1] = 5.3917;
      a.v[2] = 75.6400;
      a.v[3] = 122.4543;
      break;
    case 6:  // C: [He] 2s^2 2p^2
      a.v[1] = 11.2603;
      a.v[2] = 24.3833;
      a.l_fact[1] = a.l_fact[2] = 3;
      a.v[3] = 47.8878;
      a.v[4] = 64.4939;
      a.v[5] = 392.087;
      a.v[6] = 489.993;
      break;
    case 7:  // N: [He] 2s^2 2p^3
      a.v[1] = 14.53;
      a.v[2] = 29.601;
      a.v[3] = 47.449;
      a.l_fact[1] = a.l_fact[2] = a.l_fact[3] = 3;
      a.v[4] = 77.473;
      a.v[5] = 97.89;
      a.v[6] = 552.07;
      a.v[7] = 667.046;
      break;
    default:
      return false;
  }
  for (int i = 1; i <= an; ++i) {
    a.v_norm[i] = a.v[i] / v_h;
    a.e_c[i] = a.v_norm[i] * a.v_norm[i] / (16. * (double)i);
    a.nstar[i] = (double)i / std::sqrt(a.v_norm[i]);
    a.vfact[i] = (a.v_norm[i]) * std::sqrt(a.v_norm[i]);
    a.e_b[i] = 2. * a.vfact[i] / (3. * (2. * a.nstar[i] - 1.));
  }
  for (int i = 1; i <= an; ++i) {
    a.c_nstar[i] = std::pow(2. * euler / a.nstar[i], 2 * a.nstar[i]);
    a.c_nstar[i] = a.c_nstar[i] * (double)a.l_fact[i] / (2. * pig * a.nstar[i]);
    a.c_nstar[i] = 0.5 * a.v_norm[i] * a.c_nstar[i];
  }
  return true;
}
}  // namespace

int build_ionization_table(int an, int z0, int model, double e_max, double dt, double* tab, double* de_inv_out) {
  const double omega_a = 41.3, pig = 3.141592653589793, tiny = 1.e-10;
  const int n_ge = kNge;
  Adk a;
  if (!adk_coeff(an, a)) return -1;
  if (z0 < 0 || z0 > an || model < 1 || model > 5 || !(e_max > 0.0)) return -1;
  const int zm = an;
  const int nrow = n_ge + 2;
  std::vector<double> wi((size_t)(n_ge + 1) * (zm + 1), 0.0);
  double dge = e_max / (double)n_ge;
  double de_inv = 1. / dge;
  for (int k = z0 + 1; k <= zm; ++k) {
    int j = k - z0;
    double ns = 2. * a.nstar[k] - 1.;
    for (int i = 1; i <= n_ge; ++i) {
      double ei = dge * (double)i;
      double fact2 = (2. * a.vfact[k] / ei);
      double fact1, w_adk, w_bsi, efact, avg_fact;
      double w = 0.0;
      switch (model) {
        case 1:  // ADK DC
          fact1 = std::pow(fact2, ns);
          w_adk = a.c_nstar[k] * fact1 * std::exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          break;
        case 2:  // ADK AC = <W_DC>
          fact1 = std::pow(fact2, ns);
          fact1 = fact1 * std::sqrt(3. * ei / (pig * a.vfact[k]));
          w_adk = a.c_nstar[k] * fact1 * std::exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          break;
        case 3:  // BSI + ADK(AC)
        case 5:  // cycle-averaged BSI + ADK
          if (model == 3) {
            fact1 = std::pow(fact2, ns);
            fact1 = fact1 * std::sqrt(3. * ei / (pig * a.vfact[k]));
          } else {
            fact1 = std::sqrt(3. * ei / (pig * a.vfact[k])) * std::pow(fact2, ns);
          }
          w_adk = a.c_nstar[k] * fact1 * std::exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          if (ei > a.e_c[k]) {
            fact2 = (2. * a.vfact[k] / a.e_c[k]);
            if (model == 3) {
              fact1 = std::pow(fact2, ns);
              fact1 = fact1 * std::sqrt(3. * a.e_c[k] / (pig * a.vfact[k]));
            } else {
              fact1 = std::sqrt(3. * a.e_c[k] / (pig * a.vfact[k])) * std::pow(fact2, ns);
            }
            w_adk = a.c_nstar[k] * fact1 * std::exp(-fact2 / 3.);
            w_bsi = a.vfact[k] * (1. - a.e_c[k] / ei) / (4. * pig * (double)k);
            w = w_bsi + w_adk;
          }
          break;
        case 4:  // min(ADK<m>, BSI)
          fact1 = std::pow(fact2, ns);
          avg_fact = 1.0;
          if (a.l_fact[k] > 1) {
            for (int ll = 1; ll <= (a.l_fact[k] - 1) / 2; ++ll) avg_fact = avg_fact + 2. / std::pow(fact2, ll);
            avg_fact = avg_fact / a.l_fact[k];
            fact1 = fact1 * avg_fact;
          }
          fact1 = fact1 * std::sqrt(3. * ei / (pig * a.vfact[k]));
          w_adk = a.c_nstar[k] * fact1 * std::exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          efact = 1. - a.e_c[k] / ei;
          w_bsi = a.vfact[k] * efact / (4. * pig * (double)k);
          if (w_bsi < tiny) w_bsi = 0.;
          if (ei > a.e_c[k]) w = (w_bsi < w_adk) ? w_bsi : w_adk;
          if (ei > a.e_b[k]) w = w_bsi;
          break;
      }
      wi[(size_t)i + (size_t)(n_ge + 1) * j] = w;
    }
  }
  double dt_fs = 10. * dt / 3.;
  for (auto& x : wi) x = omega_a * x;
  std::memset(tab, 0, sizeof(double) * (size_t)nrow * (zm + 1));
  int zm_loc = zm - z0;
  for (int z = 0; z <= zm_loc - 1; ++z) {
    int zk = z + 1;
    int k = z + z0;
    for (int i = 1; i <= n_ge; ++i)
      tab[(size_t)i + (size_t)nrow * k] = 1. - std::exp(-dt_fs * wi[(size_t)i + (size_t)(n_ge + 1) * zk]);
  }
  *de_inv_out = de_inv;
  return 0;
}

}  // namespace agpu

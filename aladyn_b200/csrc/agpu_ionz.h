// agpu_ionz.h — host ADK table builder (see agpu_ionz.cpp).
#pragma once

namespace agpu {
constexpr int kNge = 10000;  // n_ge, src/ionization/ionz_data.f90:55
// Fills tab[(n_ge+2) * (an+1)] column-major (nk, z); returns 0 on success.
int build_ionization_table(int an, int z0, int model, double e_max, double dt, double* tab, double* de_inv_out);
}  // namespace agpu

// ORACLE (test infrastructure only): the level record of oracle_restrict.cpp,
// shared with the multi-level trend of oracle_trisk.cpp.
#pragma once
#include <cstdint>

extern "C" {
struct orc_rlevel {
  int n, P;
  int64_t NN;
  const double *hex_inv, *overl_a, *overl_split, *rf_wgt;  // [NN], [4*NN], [2*NN], [3*NN]
  const int64_t* hn;
  int64_t nhn;
  const int64_t* he;
  int64_t nhe;
  const int32_t *mask_n, *mask_e;                            // [NN], [3*NN]
  double *scal, *dscal, *flux, *dvelo;                       // [nz][NN], [nz][NN], [nz][3*NN], [nz][3*NN]
};
int orc_restrict_scalar(const orc_rlevel* par, const orc_rlevel* chd, int nz);
int64_t orc_restrict_flux(const orc_rlevel* par, const orc_rlevel* chd, int nz);
int orc_restrict_u_source(const orc_rlevel* par, const orc_rlevel* chd, int nz);
}

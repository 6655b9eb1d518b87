// sfd_setup.h -- host-side set-up helpers of the FDTD engine.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "sfd_internal.h"

namespace sfd {

bool holberg(int fdorder, int maxrelerror, double hc[6]);
double literal9(double v);
bool cpml_profiles(double npower, double kmax, double fpml, double vppml, double dh, double dt, int nab, float *K,
                   float *a, float *b, float *Kh, float *ah, float *bh);
void cerjan_taper(double abpc, int nab, float *taper);
int nbnd_cells(int nd, int nz, int ny, int nx, int F, int nab, int freesurf);
int transform_model(const sfd_config &c, int nz, int ny, int nx, const float *const *params,
                    std::vector<float> out[NPAR], std::string &err);
int source_targets(int nd, int mask, int type, int fields[3], float div[3]);
void point_cell(const float *pos, double DH, int F, int &i, int &j, int &k);

}  // namespace sfd

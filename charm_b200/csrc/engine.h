// Host runtime of charm_b200: device context, buffer and plan caches, and
// the call flows of grid synthesis, scattered synthesis and grid analysis.
// Used by capi.cpp; independent of any framework (plain CUDA runtime and
// cuFFT).
#pragma once

#include <string>

#include "../../include/charm_b200.h"

namespace cb
{

// Result of an engine call: CHARM_SUCCESS or a CHarm error code with a
// message.
struct Status
{
    int code = CHARM_SUCCESS;
    std::string msg;
    bool ok() const { return code == CHARM_SUCCESS; }
};

// Synthesis at grids or scattered points.  kgrad: 0 single quantity
// (dr, dlat, dlon), 1 full grad1, 2 full grad2.  f[q] receive the output
// components in CHarm's computation order (the caller reorders pointers).
Status shs_point(const charm_point *pnt, const charm_shc *shcs,
                 unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                 double **f);

// Analysis on GL/DH grids; overwrites shcs->c, shcs->s.
Status sha_point(const charm_point *pnt, const double *f, unsigned long nmax,
                 charm_shc *shcs);

// Quadrature grid nodes and weights on the GPU (north to south).
Status quad_nodes(int type, unsigned long nmax, double *lat, double *w);

// Releases all device memory and plans (called at process exit).
void shutdown();

} // namespace cb

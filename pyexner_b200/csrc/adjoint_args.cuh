// Arguments of the reverse-mode kernels (adjoint.cuh), shared with the host code.
#pragma once
#include <stdint.h>

#include "pxb_device.cuh"

namespace pxb {

struct AdjArgs {
    int ny, nx;
    long long pitch;
    double dx;
    const double *h, *hu, *hv, *zb, *z, *nb, *G;  // stage input U
    const double* h1;                              // depth after the hydro update, before the handlers
    const double *sh, *shu, *shv, *szb, *sG;      // state after handlers 1 and the grass factor
    const uint8_t* nodata;
    const double* dt;
    SedTable<double> sed;
    int mpm;
    double *Sh, *Shu, *Shv, *Szb, *SG;  // adjoint of the stage output (then of the state after handlers 2)
    double *Th, *Thu, *Thv, *Tzb, *TG;  // adjoint of the state entering the Exner update
    double *Ih, *Ihu, *Ihv, *Izb, *IG;  // adjoint of the stage input (accumulated)
    double* dtbar;                      // accumulated adjoint of dt
    // parameter adjoints (null: not requested)
    double* nbbar;  // plane: adjoint of the static n_b (friction of the Roe faces), accumulated
    double* tbar;   // MPM table of the one sediment class: np2, sm1d, thc, np3sg, sm1, frac, 1 - porosity
};

// Field slots as BcArgs: 0 h, 1 hu, 2 hv, 3 z_b, 4 n (not carried), 5 G.
struct AdjBcArgs {
    double* f[6];
    const long long* cells;
    const long long* donors;
    int count, kind;
    double nx, ny;
    double c0, c1;  // ZeroMomentum values (NaN: identity)
    double* tmp;    // 6 * count
    double vx, vy;  // ConstantInflux: d(hu, hv) / d values[0] = (values[1], values[2])
    double* qbar;   // ConstantInflux: adjoint of its values[0] (accumulated; null: not requested)
};

struct AdjCflArgs {
    int ny, nx;
    long long pitch;
    const double *h, *hu, *hv, *G;
    const uint8_t* nodata;
    double dx, cfl, floor_dt;
    unsigned long long* maxbits;
    unsigned int* nties;
    const double* dtbar;
    double *Ah, *Ahu, *Ahv, *AG;  // adjoint of the step input (accumulated)
};

}  // namespace pxb

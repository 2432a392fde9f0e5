// Host-side set-up tables of the radiation path (RADSETUP replacement).
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace mgcm {

constexpr int NV = 7, NI = 5, NG = 17, NGK = 16, NT = 7, NP11 = 11, NP = 51, NH = 10;
constexpr int NPLANCK = 8501;

struct HostTables {
    // reference layout, Fortran order: co2v(nt,np,nh,nw,ng), co2i(...)
    std::vector<double> co2v, co2i;
    std::vector<double> planckir;  // planckir(nw, it): [it*5 + nw]
    double fzerov[NV], fzeroi[NI];
    double pfgasref[NP], tgasref[NT], pgasref[NP11];
    double solarf[NV], tauray[NV], dwni[NI], dwnv[NV];
    double gweight[NG], wrefh2o[NH];
    // Largest pressure p with log10(p) <= pfgasref[n] under the host libm:
    // the bin search of tpindex done as a pressure comparison (bit-exact bins).
    double plimit[NP];
};

// Reads the two k-coefficient files (code/laginterp.f90:59-69). 0 or <0.
int read_ktables(const std::string &dir, std::vector<double> &co2v8, double fzerov[NV],
                 std::vector<double> &co2i8, double fzeroi[NI]);

// setspv/setspi/setrad/laginterp.
void build_tables(HostTables &t, const std::vector<double> &co2v8, const double fzerov[NV],
                  const std::vector<double> &co2i8, const double fzeroi[NI]);

int load_tables(const std::string &dir, HostTables &t);

// Aerosol optics tables (code/initcld.f:141-190, code/setrad.f90:73-105).
constexpr int NBIN_RT = 20, NRATIO = 15;
struct AerosolTables {
    double radb[NBIN_RT + 1];                 // radb_rt: bin boundaries (m)
    // Mie tables (REAL*4 in the reference), [quantity qext,qscat,g][bin][band]
    double dst_v[3][NBIN_RT][NV], dst_i[3][NBIN_RT][NI];
    // water-ice coated spheres, [quantity][core ratio][bin][band]
    double cld_v[3][NRATIO][NBIN_RT][NV], cld_i[3][NRATIO][NBIN_RT][NI];
    double cor_ratio[NRATIO];                 // REAL*4 core-to-mantle radius ratios
    // prescribed dust (ini_optdst via setrad): per-band QEXT, QSCAT, G
    double qextv[NV], qscatv[NV], gv[NV], qexti[NI], qscati[NI], gi[NI];
};

// Reads the dust and water-ice Mie tables and builds the bins.  0 or <0.
int load_aerosol_tables(const std::string &dir, AerosolTables &a);

// Device k-table layout: [nw][nt][np][nh][ng 0..15], Gauss point fastest.
void gauss_fastest(const HostTables &t, std::vector<double> &kv, std::vector<double> &ki);

}  // namespace mgcm

// sfref.cpp -- drives SFbox 2.1 built from the reference's own sources and
// writes its results at full precision.  Test infrastructure: the oracle's
// parity tests compare the restatement and the CUDA path with these numbers.
//
//   sfref eval  <input.in> <x.bin|-> <out.txt>    one residual evaluation
//   sfref solve <input.in> <x0.bin|-> <out.txt>   SF_Solve::Iterate from x0
//   sfref poisson <input.in> <in.bin> <out.txt>   the lattice's Poisson sweep
//                                                  and E^2 on given profiles
//
// x.bin holds the iteration variables as raw little-endian doubles in
// SF_Solve's packing; "-" keeps SFbox's own initial guess
// (SF_System::SetInitialGuess, SF_System.cpp:242-258).  The first calculation
// of the input file is run, set up as SF_Box.cpp's Go() does (SF_Box.cpp:
// 139-177) and solved as SF_System::Go does (SF_System.cpp:187-235) without
// writing SFbox's output files.
//
// out.txt has one record per line, "<key> <count> <values...>", values
// printed with 17 significant digits (exact round trip):
//   nvar, x, g (residual at x), iterations, accuracy, F, Omega,
//   state_<name>_phi, state_<name>_swf, mol_<name>_lngn, mol_<name>_phibulk,
//   (charged systems) psi, charge, epsav,
//   mol_<name>_theta, mol_<name>_phi, mol_<name>_seg_<segname>_phi
// standard and fenk headers first, so only the reference's classes see the
// access override that lets this driver read SF_Solve's iterate
#include <cstdio>
#include <deque>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>
#include <pthread.h>
#include <omp.h>
#include "fenk.h"
#define protected public
#define private public
#include "SF_Box.h"
#include "SF_System.h"
#include "Vary.h"
#undef protected
#undef private

#include <cstdio>
#include <string>
#include <vector>

SF_System *NewSystem(Input *MyInput, Boolean compute);
extern Boolean silent;
extern Boolean warnings;

static FILE *g_out;

static void put(const std::string &key, const double *v, int n) {
    fprintf(g_out, "%s %d", key.c_str(), n);
    for (int i = 0; i < n; i++) fprintf(g_out, " %.17g", v[i]);
    fputc('\n', g_out);
}
static void put1(const std::string &key, double v) { put(key, &v, 1); }
static void putv(const std::string &key, const Vector &v) {
    std::vector<double> a;
    for (int i = v.Lowerbound(); i <= v.Upperbound(); i++) a.push_back(v[i]);
    put(key, a.data(), (int)a.size());
}

static std::vector<double> read_x(const char *path) {
    std::vector<double> x;
    FILE *f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "sfref: cannot open %s\n", path);
        exit(2);
    }
    double d;
    while (fread(&d, sizeof d, 1, f) == 1) x.push_back(d);
    fclose(f);
    return x;
}

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: sfref eval|solve|poisson <input.in> <x.bin|-> <out.txt>\n");
        return 2;
    }
    const std::string mode = argv[1];
    silent = true;
    warnings = false;
    Input *MyInput = new Input(Copy(argv[2]));
    Array<Text> firstArguments(1, 10);
    firstArguments[1] = "lat";
    firstArguments[2] = "mon";
    firstArguments[3] = "state";
    firstArguments[4] = "mol";
    firstArguments[5] = "newton";
    firstArguments[6] = "output";
    firstArguments[7] = "sys";
    firstArguments[8] = "reaction";
    firstArguments[9] = "var";
    firstArguments[10] = "alias";
    MyInput->SetAllMessagesOff();
    MyInput->CheckFirstArguments(firstArguments);
    if (!MyInput->NextCalculation()) {
        fprintf(stderr, "sfref: no calculation in %s\n", argv[2]);
        return 2;
    }
    Vary *variate = new Vary(MyInput);
    variate->NextCalculation();
    SF_System *Sys = NewSystem(MyInput, true);
    Sys->SetInitialGuess(Sys, Sys->GetLattice());
    SF_Solve *Solve = Sys->GetSolve();
    const int n = Solve->GetNumItVar();
    if (mode == "poisson") {
        // the lattice's Poisson sweep and field alone: x.bin holds psi0, the
        // dielectric profile and the charge (M values each); out.txt gets
        // psi (from zeros) and E^2 (from zeros) with the preFactors
        // SF_SegmentList::ComputeElectricPotential(psi0) and
        // SF_Solve::UpdateSWF pass
        Lattice *Lat = Sys->GetLattice();
        const int M = Lat->GetTotalNumLayers();
        std::vector<double> in = read_x(argv[3]);
        if ((int)in.size() != 3 * M) {
            fprintf(stderr, "sfref: poisson wants %d values, %s holds %zu\n", 3 * M, argv[3], in.size());
            return 2;
        }
        Vector psi0(1, M), psi0b(1, M), eps(1, M), charge(1, M), psi(1, M), esq(1, M);
        for (int z = 1; z <= M; z++) {
            psi0[z] = psi0b[z] = in[z - 1];
            eps[z] = in[M + z - 1];
            charge[z] = in[2 * M + z - 1];
        }
        const double pfp = (ELEM_CHARGE / EPS0) / Lat->GetSiteDistance();
        const double pfe = (EPS0 * Lat->GetSiteDistance()) / (BOLTZMANN * TEMPERATURE);
        Lat->ElectricPotential(psi, psi0, eps, charge, pfp);
        Lat->ElectricFieldSquared(esq, psi0b, pfe);
        g_out = fopen(argv[4], "w");
        if (!g_out) return 2;
        putv("psi", psi);
        putv("esq", esq);
        Vector sites(1, M);
        for (int z = 1; z <= M; z++) sites[z] = Lat->GetNumLatticeSites(z);
        putv("sites", sites);
        fclose(g_out);
        return 0;
    }
    if (std::string(argv[3]) != "-") {
        std::vector<double> x0 = read_x(argv[3]);
        if ((int)x0.size() != n) {
            fprintf(stderr, "sfref: %s holds %zu values, the system has %d iteration variables\n", argv[3],
                    x0.size(), n);
            return 2;
        }
        for (int i = 1; i <= n; i++) Solve->x[i] = x0[i - 1];
    }
    if (mode == "solve") {
        Solve->Iterate();
    } else if (mode != "eval") {
        fprintf(stderr, "sfref: unknown mode %s\n", argv[1]);
        return 2;
    }
    std::vector<double> g(n > 0 ? n : 1);
    Solve->residuals(g.data(), &Solve->x[1]);

    g_out = fopen(argv[4], "w");
    if (!g_out) {
        fprintf(stderr, "sfref: cannot write %s\n", argv[4]);
        return 2;
    }
    put1("nvar", n);
    put("x", &Solve->x[1], n);
    put("g", g.data(), n);
    put1("iterations", Solve->getiterations());
    put1("accuracy", Solve->getaccuracy());
    SF_SegmentList *SegQ = Sys->GetSegmentList();
    SF_MoleculeList *MolQ = Sys->GetMoleculeList();
    for (int i = 1; i <= SegQ->GetNumStates(); i++) {
        SF_State *St = SegQ->GetState(i);
        std::string nm = St->GetName().str();
        putv("state_" + nm + "_phi", St->GetPhi());
        putv("state_" + nm + "_swf", St->GetSWF());
    }
    for (int m = 1; m <= MolQ->GetNumMolecules(); m++) {
        SF_Molecule *Mol = MolQ->GetMolecule(m);
        std::string nm = Mol->GetName().str();
        put1("mol_" + nm + "_lngn", Mol->GetLnGN());
        put1("mol_" + nm + "_phibulk", Mol->GetPhiBulk());
        put1("mol_" + nm + "_theta", Mol->GetTheta());
        putv("mol_" + nm + "_phi", Mol->GetPhi(total));
        SF_MolStructure *Chain = Mol->GetMolStructure();
        for (int k = 1; k <= Chain->GetNumDiffSegments(); k++) {
            SF_MolSegment *Seg = Chain->GetDiffSegment(k);
            putv("mol_" + nm + "_seg_" + Seg->GetName().str() + "_phi", Seg->GetPhi(total));
        }
    }
    put1("F", MolQ->GetFreeEnergy());
    put1("Omega", MolQ->GetGrandPotential());
    if (SegQ->Charged()) {
        putv("psi", SegQ->GetElectricPotential());
        putv("charge", SegQ->GetCharge());
        putv("epsav", SegQ->GetAverageEpsilon());
    }
    fclose(g_out);
    return 0;
}

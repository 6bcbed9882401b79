// c1_residual.cpp -- a C++ caller of include/sfgpu.h, built the way a
// maintainer would bind SFbox to the library: it fills the descriptors as
// an SF_Solve constructor would for the C1 input (Lat1DFlat1stO, 100 layers,
// surface / mirror1, lambda 1/6, frozen S at the surface, (A)100 free at
// phibulk 0.01 in solvent W, chi_AW 0.5, chi_AS -1.0), evaluates one residual
// through sfgpu_residual_host and writes f.
//
//   c1_residual <x.bin> <f.bin>      (raw little-endian doubles, 200 each)
#include <cstdio>
#include <vector>

#include "sfgpu.h"

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: c1_residual <x.bin> <f.bin>\n");
        return 2;
    }
    int ndev = 0;
    if (sfgpu_device_count(&ndev) != SFGPU_OK || ndev < 1) {
        std::fprintf(stderr, "no device: %s\n", sfgpu_last_error());
        return 3;
    }
    const int n = 100, M = n + 2;

    sfgpu_lattice_desc L = {};
    L.gradients = 1;
    L.geometry = SFGPU_GEOM_FLAT;
    L.order = 1;
    L.n_layers[0] = n;
    L.bound_lo[0] = SFGPU_BOUND_SURFACE;
    L.bound_hi[0] = SFGPU_BOUND_MIRROR1;
    L.lambda = 1.0 / 6.0;
    L.lambda_chi = -1;
    L.layer_adjustment = 1;
    L.dimensions = 3;
    L.offset_first_layer = 0;
    L.stiff_range = nullptr;
    L.lattice_type = SFGPU_LATTICE_STANDARD;

    // states in input order S, A, W; S frozen on the lower boundary layer
    std::vector<double> surface(M, 0.0);
    surface[0] = 1.0;
    std::vector<sfgpu_segment_desc> segs(3);
    segs[0].freedom = SFGPU_SEG_FROZEN;
    segs[0].range = surface.data();
    segs[1].freedom = SFGPU_SEG_FREE;
    segs[1].range = nullptr;
    segs[2].freedom = SFGPU_SEG_FREE;
    segs[2].range = nullptr;
    std::vector<double> chi(9, 0.0);
    chi[1 * 3 + 2] = chi[2 * 3 + 1] = 0.5;    // A - W
    chi[1 * 3 + 0] = chi[0 * 3 + 1] = -1.0;   // A - S

    const int pol_seg[1] = {1}, pol_len[1] = {100};
    const int w_seg[1] = {2}, w_len[1] = {1};
    std::vector<sfgpu_molecule_desc> mols(2);
    mols[0] = sfgpu_molecule_desc{1, pol_seg, pol_len, SFGPU_MOL_FREE, 0.01, 0.0, 0, nullptr, nullptr, 0.0, nullptr, 0};
    mols[1] = sfgpu_molecule_desc{1, w_seg, w_len, SFGPU_MOL_SOLVENT, 0.0, 0.0, 0, nullptr, nullptr, 0.0, nullptr, 0};

    sfgpu_system_desc D = {L, (int)segs.size(), segs.data(), chi.data(), nullptr,
                           (int)mols.size(), mols.data(), 0};
    sfgpu_system *gpu = nullptr;
    if (sfgpu_system_create(&D, &gpu) != SFGPU_OK) {
        std::fprintf(stderr, "sfgpu_system_create: %s\n", sfgpu_last_error());
        return 4;
    }
    int m = 0, nvar = 0, nclass = 0, nsites = 0;
    sfgpu_system_info(gpu, &m, &nvar, &nclass, &nsites);
    std::vector<double> x(nvar), f(nvar);
    FILE *fx = std::fopen(argv[1], "rb");
    if (!fx || std::fread(x.data(), sizeof(double), x.size(), fx) != x.size()) {
        std::fprintf(stderr, "cannot read %d values from %s\n", nvar, argv[1]);
        return 5;
    }
    std::fclose(fx);
    if (sfgpu_residual_host(gpu, x.data(), f.data()) != SFGPU_OK) {
        std::fprintf(stderr, "sfgpu_residual_host: %s\n", sfgpu_last_error());
        return 6;
    }
    double F = 0;
    sfgpu_free_energy(gpu, &F);
    FILE *ff = std::fopen(argv[2], "wb");
    std::fwrite(f.data(), sizeof(double), f.size(), ff);
    std::fwrite(&F, sizeof(double), 1, ff);
    std::fclose(ff);
    sfgpu_system_destroy(gpu);
    std::printf("M %d nvar %d F %.17g\n", m, nvar, F);
    return 0;
}

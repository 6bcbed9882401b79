// sfgpu_system.h -- host object behind the opaque sfgpu_system handle.
#pragma once
#include <vector>
#include "sfgpu_logspace.cuh"
#include "sfgpu_charge.cuh"

struct HostLat {
    DLat L;
    std::vector<double> lam_m, lam_p, lamc_m, lamc_p, Lx, w_gn, w_f;
    std::vector<double> sb;   // SubtractBoundaries factors (0 removed, 1/2 mirror2 layers)
    std::vector<double> stiff; // 'lat : stiff_range' mask (3D second order), empty if none
};
int sfgpu_build_lattice(const sfgpu_lattice_desc *d, HostLat *H);
// weights of a constant-force step with force f (see sfk::force_row)
sfk::ForceW force_weights(const DLat &L, double f);

struct HMol {
    int N = 0, type = 0, sym = 0, freedom = 0, pinned = 0;
    double phibulk = 0, theta = 0, chemintref = 0;
    std::vector<int> seg, used, count;
    // symmetric dendrimer (SF_Dend1stO): per generation its positions'
    // segments (first = branch point) and functionality; nshort = positions
    // from the centre to an end
    int dend = 0, nshort = 0;
    double force = 0;                 // mol : force (constant-force ensemble)
    // branched molecule: parent[s] of every segment (parent[0] = -1,
    // parent[s] < s) and the children of every segment in increasing order
    int tree = 0;
    std::vector<int> parent;
    std::vector<std::vector<int>> kids;
    // a symmetric dendrimer written out as its bond tree (tseg, tparent,
    // tkids; built by the derivatives, which run the tree recursion on it)
    std::vector<int> tseg, tparent;
    std::vector<std::vector<int>> tkids;
    int ring = 0;                     // homopolymer ring (SF_HomoRing1stO)
    double ring_norm0 = 0;            // return weight of the free ring (NORM[0])
    std::vector<std::vector<int>> gen_seg;
    std::vector<int> gen_rep;
    std::vector<double *> d_phi;      // per segment (used ones)
    std::vector<double *> d_dphi;     // tangents (allocated on first J*v)
    std::vector<double *> d_ori;      // bond orientation per segment, mphi*M (when enabled)
};

struct sfgpu_system {
    HostLat H;
    int M = 0, K = 1, nseg = 0, nmol = 0, nclass = 0, nsites = 0, solvent = -1;
    size_t nvar = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<double> chi, pf, range_h;
    std::vector<int> freedom, class_of, rep_of_class, sites_h;
    std::vector<HMol> mols;
    sfk::BulkParam bp;
    ChiTable ct;
    // device buffers
    double *d_lam_m = nullptr, *d_lam_p = nullptr, *d_lamc_m = nullptr, *d_lamc_p = nullptr;
    double *d_wgn = nullptr, *d_wf = nullptr, *d_sb = nullptr, *d_stiff = nullptr;
    int *d_jmap = nullptr, *d_sites = nullptr;
    std::vector<double *> d_range, d_gfull, d_gseg, d_phi;
    double *d_gi = nullptr, *d_ginv[2] = {nullptr, nullptr};
    double *d_partial = nullptr, *d_scal = nullptr, *d_phib = nullptr, *d_chib = nullptr, *d_misc = nullptr;
    double *d_x = nullptr, *d_f = nullptr;
    int nblocks_red = 1;
    // 3D first-order step, separately for the composition-free forward steps
    // and the composing backward steps: x planes per block and whether the
    // software-pipelined form (step3d_march_pf) runs it
    int tile_xc = 4, tile_xc_bwd = 8;
    int tile_pipelined = 0, tile_pipelined_bwd = 1;
    // chain storage of residual evaluations: 0 keeps every forward slice,
    // k > 0 keeps every k-th one and recomputes the others segment by
    // segment during the backward sweep (set at creation)
    int primal_stride = 0;
    bool primal_checkpointed(const HMol &o) const;
    // bond-orientation profiles of second-order lattices (off by default)
    bool orient = false;
    double *d_ori_sum = nullptr;
    int mphi() const { return K == 3 ? 2 : 3; }
    int set_orientation(int enable);
    // forward-mode tangent buffers, allocated on the first J*v
    bool t_ready = false;
    std::vector<double *> dgfull, dgseg, dphi;
    double *d_dgi = nullptr, *d_dginv[2] = {nullptr, nullptr};
    // the tangent's chain storage (every position): the primal's d_gi, or a
    // buffer of its own when the primal keeps checkpoints only; two work
    // slices for the steps whose tangent is formed from two primal steps
    double *t_gi = nullptr, *t_w[2] = {nullptr, nullptr};
    double *d_tscal = nullptr, *d_dpartial = nullptr, *d_dphib = nullptr, *d_dchib = nullptr;
    double *d_v = nullptr, *d_jv = nullptr;
    int ensure_tangent();
    int molecule_phi_t(int m);
    int jvp_async(const double *x, const double *v, double *f, double *jv);
    // reverse-mode (adjoint) buffers, allocated on the first J^T w
    bool a_ready = false;
    double *a_gf = nullptr, *a_gb = nullptr, *a_cot[2] = {nullptr, nullptr};
    // chain storage of the reverse sweep: every slice (a_stride 0) or
    // checkpoints every a_stride positions plus two segment buffers
    int a_stride = 0;
    bool a_misc = false;
    double *a_store = nullptr;
    double *a_ring = nullptr;               // ring walk levels of the reverse sweep (ring_phi_adj)
    size_t a_ring_doubles = 0;
    double *a_tree = nullptr;               // bond-tree cotangents (molecule_adjoint_tree)
    size_t a_tree_doubles = 0;
    int molecule_adjoint_tree(int m);
    // slices of the bond-tree recursion: d_gi, or while a dendrimer runs as
    // its tree in the reverse sweep (3N slices) a_dend_gi
    double *tree_gi = nullptr;
    double *a_dend_gi = nullptr;
    size_t a_dend_gi_doubles = 0;
    void build_dend_tree(HMol &o);
    void dend_view(HMol &o, bool on);
    double *a_ckF = nullptr, *a_ckB = nullptr, *a_bufF = nullptr, *a_bufB = nullptr;
    int a_qseg = -1;                        // segment held in a_bufF / a_bufB
    std::vector<double *> a_phibar, a_gbar, a_phibar_raw;
    double *a_scal = nullptr, *a_chibbar = nullptr, *a_qbar = nullptr, *a_w = nullptr, *a_xbar = nullptr;
    int ensure_adjoint();
    int ensure_adjoint_misc();
    int store_chains(int m, bool compose, const double **gb0);
    int store_chains_ck(int m, bool compose, const double **gb0);
    int load_segment(int m, int q);
    void adj_start(const double *G, double *dst);
    void adj_fstep(const HMol &o, int t, const double *src, double *dst);
    void adj_bstep(const HMol &o, int t, const double *src, double *dst, const double *other, double *phi);
    int set_checkpoint(int stride);
    int molecule_phi_store(int m);
    int molecule_adjoint(int m, double *const *phibar_src);
    int primal_store(const double *x, double *f);
    int free_energy_grad(const double *x, double *F, double *xbar);
    int phi_vjp_async(const double *x, const double *const *omega, double *xbar);
    int chi_vjp_async(const double *x, const double *w, double *dchi);
    std::vector<double *> a_phibar_m;
    int vjp_async(const double *x, const double *w, double *f, double *xbar);
    int launch_step1(const double *gin, const double *G, double *gout, const double *other, double *phi, int mode);
    // overflow protection: chain statistics in logarithms (first-order 1D/2D)
    bool logmode = false;
    sfk::LogLat logq;
    sfk::LogConst logc;
    std::vector<double> w_os;                 // lnGN weights of the log-space lattices
    double *d_wos = nullptr, *d_lse = nullptr;
    double *d_logl0x = nullptr, *d_loglmx = nullptr, *d_loglpx = nullptr;
    std::vector<double *> d_lgseg;            // log G per segment (MakeSafe)
    int setup_logspace();
    int molecule_phi_log(int m);
    int molecule_phi_dend(int m);
    int molecule_phi_tree(int m);
    int molecule_phi_ring(int m);
    // charges (1D flat): valence and dielectric constant per segment, the
    // neutralizer molecule, psi0/psi/E^2 and the iteration layout
    bool charged = false;
    int neutralizer = -1;
    std::vector<double> valence, epsilon;
    sfk::QParam qp;
    double *d_neut_phib = nullptr, *d_el = nullptr, *d_surf = nullptr;
    int setup_charges(const sfgpu_system_desc *d, const std::vector<int> &jmap);
    std::vector<void *> allocs;

    ~sfgpu_system();
    int alloc_d(double **p, size_t n);
    int alloc_i(int **p, size_t n);
    int setup(const sfgpu_system_desc *d);
    int molecule_phi(int m);
    int residual_async(const double *x, double *f);
    int free_energy(double *F);
    int thermo(double *F, double *Omega, double *fe, double *gp);
};

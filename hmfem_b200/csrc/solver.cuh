// solver.cuh -- the solver object behind the hmfem_* C-ABI.
#pragma once
#include <type_traits>
#include <vector>

#include "hm.cuh"

namespace hm {

template <class T> struct Seed;  // cycle.cuh
struct Demote;                     // cycle.cuh

struct Solver {
    hmfem_options opt;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    AllocCache *cache = nullptr;

    // grid problem (hmfem_assemble)
    bool have_grid = false;
    int nx = 0, ny = 0, nz = 0;
    double hx = 0, hy = 0, hz = 0, visc = 1;
    int bc[6] = {0, 0, 1, 1, 1, 1};
    const double *KX = nullptr, *KY = nullptr, *KZ = nullptr;
    double *Kown[3] = {nullptr, nullptr, nullptr};
    double *face[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double *mm = nullptr;  // flux min / max

    // level-0 matrix and right-hand side
    double *b = nullptr;
    std::vector<Level> lv;
    int nlevels = 0;
    bool setup_done = false;
    bool bad_matrix = false;  // the last assembly met an invalid permeability
    bool l0_same = false;  // the last matrix set equals the one setup used
    int direct_level = -1;
    double *dense_L = nullptr;

    // CG state
    double *x = nullptr, *r = nullptr, *s = nullptr, *v = nullptr, *z = nullptr;
    // set while the CG applies the FP32 V-cycle: the level-0 prolongation
    // of the exact reduction then also forms (z, r), (z, v) and beta
    bool fuse_zdots = false;
    bool zdots_done = false;
    Ctl *ctl = nullptr;
    Ctl ctl_init{};  // host copy of the control block a solve starts from
    Ctl *ctl_host = nullptr;  // pinned, 2 slots
    double *part = nullptr;
    int *dwork = nullptr;
    unsigned *gsbar = nullptr;  // grid barrier of the fused Gauss-Seidel sweeps
    bool ctl_active = false;
    int first_sigma = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    unsigned long long graph_kernels = 0;  // kernels in one captured iteration
    hmfem_stats last{};

    // the coupled reservoir / conduit run (karst.cu), when one was made
    struct KarstRun *karst = nullptr;

    bool use_bf16(int l) const
    {
        return opt.precision == 1 && opt.bf16_from >= 0 && l >= opt.bf16_from;
    }
    // structured solve-phase forms (stencil_cycle.cu), when setup built them
    bool use_g7(int l) const { return l == 0 && !lv.empty() && lv[0].g7.cf; }
    bool use_g19(int l) const { return l == 1 && (int)lv.size() > 1 && lv[1].g19.v; }
    // level 1 is the Schur complement of level 0's red-black split
    // (opt.schur0, FP32 cycle): level 0 is then reduced exactly
    bool schur0_built = false;
    bool use_schur0() const { return schur0_built && use_g7(0); }
    // level vectors; level 0 of the FP64 cycle works on the CG's r and z
    template <class T> T *vec_f(int l);
    template <class T> T *vec_ua(int l);
    template <class T> T *vec_ub(int l);
    template <class T> T *vec_rs(int l);
    template <class T> const T *vec_dinv(int l);  // smoother diagonal
    template <class T> const T *vec_dtrue(int l); // 1 / a_ii
    template <class T> const T *sval(int l);
};

template <> inline double *Solver::vec_f<double>(int l) { return l == 0 ? r : lv[l].f; }
template <> inline float *Solver::vec_f<float>(int l) { return lv[l].f32; }
template <> inline double *Solver::vec_ua<double>(int l) { return lv[l].ua; }
template <> inline float *Solver::vec_ua<float>(int l) { return lv[l].ua32; }
template <> inline double *Solver::vec_ub<double>(int l) { return l == 0 ? z : lv[l].ub; }
template <> inline float *Solver::vec_ub<float>(int l) { return lv[l].ub32; }
template <> inline double *Solver::vec_rs<double>(int l) { return lv[l].rs; }
template <> inline float *Solver::vec_rs<float>(int l) { return lv[l].rs32; }
template <> inline const double *Solver::vec_dinv<double>(int l) { return lv[l].dsm; }
template <> inline const float *Solver::vec_dinv<float>(int l) { return lv[l].dsm32; }
template <> inline const double *Solver::vec_dtrue<double>(int l) { return lv[l].dinv; }
template <> inline const float *Solver::vec_dtrue<float>(int l) { return lv[l].dinv32; }
template <> inline const double *Solver::sval<double>(int l) { return lv[l].S.val; }
template <> inline const float *Solver::sval<float>(int l) { return lv[l].S.val32; }

int cg_init(Solver &s, cudaStream_t st);
int cg_iteration(Solver &s, cudaStream_t st);
int cg_precondition(Solver &s, cudaStream_t st);
int cg_final_residual(Solver &s, cudaStream_t st);
int launch_smoother_diag(const Csr &A, int kind, double *dsm, float *dsm32,
                         cudaStream_t st);
int dense_factor(const Csr &A, double *Lf, int *err, cudaStream_t st);
int time_kernel(Solver &s, int which, int l, int reps, float *ms, double *bytes);
int level_spmv(Solver &s, int l, const double *x, double *y, cudaStream_t st);

// structured level-0 / level-1 kernels (stencil_cycle.cu); V is the
// coefficient storage type
template <class T, class V>
int g7_pre(const Level &L, const T *f, const T *u, T *rs, const Ctl *ctl, cudaStream_t st);
template <class T>
int g7_restrict(const Level &L, const T *rs, T *fc, Seed<T> sd, const Ctl *ctl,
                cudaStream_t st);
template <class T>
int g7_prolong(const Level &L, const T *uc, T *u, const Ctl *ctl, cudaStream_t st);
// the exact red-black reduction of level 0 (schur0): coarse right-hand side
// from f, and the level-0 result from the coarse one
template <class T>
int g7_sred(const Level &L, const T *f, const T *dinv, T *fc, Seed<T> sd, const Ctl *ctl,
            cudaStream_t st);
template <class T>
int g7_sprol(const Level &L, const T *f, const T *dinv, const T *uc, T *z, const Ctl *ctl,
             cudaStream_t st);
// g7_sprol that, where it runs as one thread per C/F pair (nx even), also
// forms the CG's (z, r), (z, v) and beta (*fused = true)
template <class T>
int g7_sprol_zd(const Level &L, const T *f, const T *dinv, const T *uc, T *z,
                const double *r, const double *v, Ctl *ctl, double *part, int first,
                bool *fused, cudaStream_t st);
template <class T, class V, bool DOT>
int g7_post(const Level &L, const T *f, const T *dinv, T w, const T *u, T *uo, Ctl *ctl,
             double *part, int first, cudaStream_t st);
int g7_spmv_dot(const Level &L, const double *x, double *y, Ctl *ctl, double *part,
                 cudaStream_t st);
int g7_resid(const Level &L, const double *b, const double *x, double *r, Ctl *ctl,
             double *part, int init, Seed<double> sd, Demote dm, cudaStream_t st);
int g7_spmv(const Level &L, const double *x, double *y, cudaStream_t st);
template <class T, class V>
int g19_pre(const Level &L, const T *f, const T *u, T *rs, const Ctl *ctl, cudaStream_t st);
template <class T, class V>
int g19_post(const Level &L, const T *f, const T *dinv, T w, const T *u, T *uo,
              const Ctl *ctl, cudaStream_t st);
int g19_spmv(const Level &L, const double *x, double *y, cudaStream_t st);

// solver.cu entry points the coupled driver (karst.cu) builds on
int setup(Solver &s);
int solve(Solver &s, const double *b, double *x, int mem, hmfem_stats *out);
int profile_iteration(Solver &s, int iters, hmfem_kernel_time *out, int cap, int *count);
int batch_solve(Solver *const *ss, int m, double *const *x, int mem, hmfem_stats *out);
// Rebuilds level 0 of the last hmfem_assemble grid (same K, faces and
// boundary types) with the karst / well exchange terms: KI, WI in the
// diagonal, WI*pw in the right-hand side (device arrays, nullable).  The
// hierarchy is dropped; the next solve sets up again.
int assemble_coupled(Solver &s, const double *KI, const double *WI, const double *pw);
void karst_release(Solver &s);  // karst.cu

}  // namespace hm

struct hmfem_solver {
    hm::Solver s;
};

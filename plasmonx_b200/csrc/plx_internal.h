// Internal declarations shared by the plasmonx_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "../../include/plasmonx_b200.h"

#define PLX_CHECK_CUDA(call)                                                   \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            throw plx::Error(PLX_ERR_CUDA, std::string(#call) + ": " +         \
                                               cudaGetErrorString(e_));        \
        }                                                                      \
    } while (0)

namespace plx {

// NVTX range over a scope: the library's phases show up by name in Nsight
// Systems timelines (no cost without a tool attached).
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

struct Error {
    plx_status code;
    std::string msg;
    Error(plx_status c, std::string m) : code(c), msg(std::move(m)) {}
};

// Vectors of complex unknowns are stored "split": the n real parts followed by
// the n imaginary parts.  A batch of C vectors [C][2][n] is then a row-major
// (2C x n) real matrix, which is the operand layout of the T contraction.
struct Cplx {
    double re, im;
};

// ---------------------------------------------------------------------------
// device memory accounting
// ---------------------------------------------------------------------------
void *dev_alloc(plx_ctx *ctx, size_t bytes);
void dev_free(plx_ctx *ctx, void *p, size_t bytes);

template <typename T>
struct DevArray {
    plx_ctx *ctx = nullptr;
    T *p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { release(); }
    void alloc(plx_ctx *c, size_t count) {
        release();
        ctx = c;
        n = count;
        p = count ? static_cast<T *>(dev_alloc(c, count * sizeof(T))) : nullptr;
    }
    void release() {
        if (p) dev_free(ctx, p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

}  // namespace plx

struct plx_ctx {
    int device = 0;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    std::string last_error;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t launches = 0;  // kernels launched by the library since creation
    // polls of every bounded pipeline wait in the tensor-core kernels before
    // they give up (plx_set_wait_limit)
    static constexpr uint32_t kDefaultWaitLimit = 1u << 22;
    uint32_t wait_limit = kDefaultWaitLimit;
    // contraction profiling (plx_profile_enable)
    bool profile = false;
    std::vector<cudaEvent_t> prof_events;   // pairs (start, stop), reused
    std::vector<int> prof_cat;              // category of each pair
    size_t prof_used = 0;                   // events in use
    static constexpr int kProfCategories = 9;  // plx_profile_read categories 0..8
    double prof_flops[kProfCategories] = {}, prof_bytes[kProfCategories] = {};
    int64_t prof_launches[kProfCategories] = {};
};

struct plx_geom {
    plx_ctx *ctx = nullptr;
    int model = 0;
    int n_atoms = 0, n_types = 0, n_var = 0;
    int rhs_potential = 0;
    double e0 = 0.0;
    // host copies of the description
    std::vector<double> coord;          // 3 x N
    std::vector<int32_t> atom_type;     // N
    std::vector<double> frac;           // n_types x N neighbour fractions
    std::vector<double> eta, r_q, r_mu, tau, density, a_ij;  // per type
    std::vector<double> fermi_d, fermi_s, r0;                // type pair
    // device: per-atom data
    plx::DevArray<double> d_pos;        // [4][N]: x, y, z, unused
    plx::DevArray<int32_t> d_type;      // N
    plx::DevArray<double> d_par;        // [4][N]: r_q, r_mu, eta, a_ij of the atom's type
    plx::DevArray<double> d_frac;       // n_types x N
    // device: conductance K in CSR (off-diagonal entries with K_ij or K_ji != 0)
    plx::DevArray<int32_t> d_rowptr;    // N + 1
    plx::DevArray<int32_t> d_col;       // nnz
    plx::DevArray<double> d_kval;       // nnz: K_ij
    plx::DevArray<double> d_ktval;      // nnz: K_ji
    int64_t nnz = 0;
    // device: dense interaction matrix T (n_var x n_var, row-major; symmetric
    // for wFQ / wFQFMu; for BEM the Green-function derivative stored transposed,
    // d_T[j][i] = D(i, j))
    plx::DevArray<double> d_T;
    bool has_T = false;
    bool t_symmetric = true;
    // BEM: tessera frame [9][n] (normal, tangent 1, tangent 2), the diagonal of D
    // before the accurate closure (IEFPCM right-hand side), S A^-1 and D S A^-1
    // (column-major, IEFPCM direct solve), solvent permittivity, z(w) per frequency
    plx::DevArray<double> d_frame, d_dpre, d_M, d_DM;
    double eps_solvent = 1.0;
    std::vector<plx::Cplx> bem_z;
    // frequencies
    int n_freq = 0;
    std::vector<double> omega;                 // n_freq
    std::vector<plx::Cplx> alpha_w;            // n_types x n_freq
    plx::DevArray<plx::Cplx> d_dq;             // n_types x n_freq: charge diagonal -z(w)
    plx::DevArray<plx::Cplx> d_inv_alpha;      // n_types x n_freq: 1 / alpha_t(w)
    plx::DevArray<plx::Cplx> d_wratio;         // n_types x n_types x n_freq: w_tj / w_ti
    // mixed precision: T split into BF16 high / low parts ([n_var][ldk], k padded
    // to a multiple of 64 with zeros), the matching split of the input columns,
    // and the error word of the tensor-core kernel
    plx::DevArray<uint16_t> d_Th, d_Tl, d_Xh, d_Xl;
    int64_t ldk = 0;
    // one atom type: the operator's frequency-independent matrix
    // A0 = blockdiag(K - P, I) T folded once and split like T, so that a
    // tensor-core application of A(w) is one contraction plus the diagonal
    plx::DevArray<uint16_t> d_Ah, d_Al;
    // rows of the folded operand: n, plus for alloys the T charge rows of the
    // interface atoms J (atoms with a neighbour of the other type, and those
    // neighbours), whose products feed the w-dependent correction
    //   y_i += sum_{j of other type} 1/2 (w_tj/w_ti - 1) K_ji (s_j - s_i)
    // over the interface rows I (CSR over I, columns as positions in J)
    int64_t fold_rows = 0;
    int n_iface = 0, n_xrows = 0;
    plx::DevArray<int32_t> d_iface_atom;          // [|J|]
    plx::DevArray<int32_t> d_xrow, d_xipos;       // [|I|]: row atom, its position in J
    plx::DevArray<int32_t> d_xrowptr;             // [|I| + 1]
    plx::DevArray<int32_t> d_xcol, d_xtj;         // position of j in J, type of j
    plx::DevArray<double> d_xkt;                  // K_ji
    plx::DevArray<double> d_fold_work;            // [R][fold_rows] output of the folded contraction
    // FP32 partial sums of the k-pieces of the tensor-core contraction's split
    // tiles ([piece][column][256 rows])
    plx::DevArray<float> d_tcpart;
    plx::DevArray<int> d_tc_err;
    // diagonal of blockdiag(Kop, I) T on the charge rows, frequency independent parts:
    // a_i = sum_j K_ij (T_ij - T_ii), b_i,t = sum_{j of type t} K_ji (T_ij - T_ii)
    plx::DevArray<double> d_diag_a, d_diag_b;
    // split-K partial sums of the few-column contraction (grown on demand;
    // used only by work ordered on the context's single stream)
    plx::DevArray<double> d_part;
    // continuous batches open on this geometry (they own its frequency table)
    int open_batches = 0;
    // Hessenberg reduction A0 = Q H Q^T of the scalar-shift models: reflectors
    // (column k below row k), their 2 / v^T v, and H row-major
    plx::DevArray<double> d_hess_v, d_hess_beta, d_hess_rows;
    // timing of the last plx_solve
    double last_ms = 0.0;
    int64_t last_launches = 0;
};

namespace plx {

// How the T contraction of an operator application is computed.
enum class Contraction : int {
    FP64 = 0,       // stored T, FP64 on the CUDA cores
    FP64_OTF = 1,   // tiles generated in the kernel, FP64
    TC3 = 2,        // stored T split in BF16 high/low, 3 tensor-core products
    TC1 = 3         // stored T rounded to BF16, 1 tensor-core product
};

// Column descriptor of a batched operator application: which frequency the
// column belongs to.
struct OpBatch {
    int count = 0;            // number of columns
    const int32_t *d_freq;    // device, [count]: frequency index of each column
};

inline bool is_bem(const plx_geom *g) { return g->model == PLX_BEM_DPCM || g->model == PLX_BEM_IEF; }

// geometry.cu
void build_conductance(plx_geom *g);
void build_dense_t(plx_geom *g);
void upload_frequency_tables(plx_geom *g);

// operator.cu
//   Y = A(w_c) X for a batch: X, Y are [count][2][n_var] split-complex, device.
//   work must hold 2*count*n_var doubles.
void apply_operator(plx_geom *g, const OpBatch &b, const double *X, double *Y, double *work,
                    Contraction how);
//   S = T X (no K, no diagonal), S and X as above.
void contract_t(plx_geom *g, int count, const double *X, double *S, Contraction how);
void rhs_batch(plx_geom *g, const OpBatch &b, const int32_t *d_pol, double *Bout);
//   1 / diag(A(w_c)) for every column, [count][2][n] split complex.
void diagonal_inverse(plx_geom *g, const OpBatch &b, double *Pinv);

// tc_contract.cu: S = T X with BF16-split operands on the tensor cores
// (nprod 3: Th Xh + Th Xl + Tl Xh; nprod 1: Th Xh).  X, S: [count][2][n] FP64.
void build_t_split(plx_geom *g);
void tc_contract(plx_geom *g, int count, const double *X, double *S, int nprod, bool folded = false);
// Several contractions (geometries of one context, same product count) in ONE
// launch: every CTA finds its contraction and tile in a table of groups.
struct TcItem {
    plx_geom *g;
    int count;
    const double *X;
    double *S;
    int nprod;
    bool folded;
};
void tc_contract_group(const std::vector<TcItem> &items);
// true when apply_operator contracts with the folded A0 on the tensor cores:
// every atomistic geometry (T stored or generated; alloys with the interface
// correction)
inline bool tc_folds_operator(const plx_geom *g) { return g->model == PLX_WFQ || g->model == PLX_WFQFMU; }
// builds the folded operand if needed; returns its number of rows
int64_t tc_fold_rows(plx_geom *g);
int tc_error(plx_geom *g);   // non-zero when a tensor-core CTA gave up waiting

// inversion.cu
// d_vars: [count][2][n] right-hand sides in, solutions of A(w_i) x = b out.
void solve_inversion_cols(plx_geom *g, int i_freq, int count, double *d_vars);

// hessenberg.cu: direct solve of the models whose frequency dependence is a
// multiple of the identity (one-type wFQ, BEM DPCM): one Hessenberg reduction
// per geometry, O(n^2) per frequency, every frequency of a call in one launch.
bool hessenberg_applies(const plx_geom *g, int cols);
void build_hessenberg(plx_geom *g);
// B, X: [freqs.size() * cols][2][n]; false when a triangular factor is singular
bool hessenberg_solve(plx_geom *g, const std::vector<int32_t> &freqs, int cols, const double *B, double *X);
// C = A B for column-major n_var x n_var FP64 matrices (cuBLAS)
void bem_dgemm(plx_geom *g, const double *A, const double *B, double *C);

// bem.cu: tesserae, the Green-function derivative D (approximate or accurate),
// the BEM operator rows (S + z x), right-hand sides and the direct-solve matrix.
// tri_host: [n][3 vertices][3] bohr.
void build_bem(plx_geom *g, const double *tri_host, double normal_factor, double sphere_r, int accurate);
void build_bem_ief(plx_geom *g);
void bem_apply_rows(plx_geom *g, const OpBatch &b, const double *S, const double *X, double *Y);
void bem_rhs(plx_geom *g, const OpBatch &b, const int32_t *d_pol, double *Bout);
void bem_diagonal_inverse(plx_geom *g, const OpBatch &b, double *Pinv);
// column-major complex A(w_i) into A (n x n)
void bem_assemble_matrix(plx_geom *g, int i_freq, double2 *A);

// gmres.cu
struct GmresRequest {
    std::vector<int32_t> freq, pol;   // per column
    int m = 0;                        // Krylov dimension
    double tol = 0.0;                 // absolute
    std::vector<double> tols;         // per-column absolute tolerance (overrides tol)
    Contraction contraction = Contraction::FP64;
    bool record_trace = false;
    // inner solve of iterative refinement: the least-squares solution is taken
    // when the residual estimate passes the tolerance or at the last step, with
    // no true-residual check (the caller forms the FP64 residual)
    bool inner = false;
    // right preconditioning by the inverse diagonal of A(w) (inner solves only):
    // the operator becomes A P^-1 and the returned correction P^-1 y
    bool jacobi = false;
    // inner solves only: Krylov basis stored in FP32, and classical Gram-Schmidt
    // without the second pass (the inner tolerance is loose and the refinement's
    // FP64 residual catches what a less orthogonal basis loses)
    bool basis_fp32 = false;
    bool single_pass = false;
};
struct GmresResult {
    std::vector<int32_t> status, steps;
    std::vector<double> trace;        // [col][m]
};
// B and X are [C][2][n] device arrays; X receives the solutions.
void gmres_batched(plx_geom *g, const GmresRequest &rq, const double *d_B, double *d_X,
                   GmresResult &res);
// An operator application a solve asks for: Y = A(w) X on the batch b of
// geometry g, with `work` scratch of the same size as X.
struct OpInput {
    plx_geom *g;
    OpBatch b;
    const double *X;
    double *Y;
    double *work;
    Contraction how;
};
// A batched GMRES advanced one Arnoldi step at a time (make_gmres has run the
// set-up): while wants_product(): pre() returns the batch to multiply, the
// caller writes its product to OpInput::Y, then post(); finally end().  B, X
// and res must outlive the stepper.
struct GmresStepper {
    virtual ~GmresStepper() = default;
    virtual bool wants_product() const = 0;
    virtual OpInput pre() = 0;
    virtual void post() = 0;
    virtual void end() = 0;
};
std::unique_ptr<GmresStepper> make_gmres(plx_geom *g, const GmresRequest &rq, const double *d_B, double *d_X,
                                         GmresResult &res);
// Several operator applications at once: the tensor-core contractions of
// folded atomistic geometries that share a context are ONE grouped launch; any
// other application runs on its own.
void apply_operator_group(const std::vector<OpInput> &items);

// refine.cu: iterative refinement -- FP64 residuals r = b - A x outside, an
// inner GMRES of dimension inner_m with `inner` contraction on A d = r to a
// relative tolerance inner_rel, x += d; stops when ||r|| < tol (absolute).
struct RefineRequest {
    std::vector<int32_t> freq, pol;
    double tol = 0.0;
    int inner_m = 64;
    double inner_rel = 1e-5;
    int max_outer = 50;
    Contraction inner_contraction = Contraction::TC3;
    Contraction outer_contraction = Contraction::FP64;
    bool jacobi = true;      // diagonal right preconditioning of the inner solves
    bool single_pass_gs = true;   // tensor-core inner solves: one classical Gram-Schmidt pass
    // inner GMRES(inner_m) cycles per outer step: a cycle that ends on the full basis
    // restarts from the inner residual (inner contraction) before an FP64 residual
    int max_cycles = 1;
};
struct RefineResult {
    std::vector<int32_t> status, inner_steps, outer;
    std::vector<double> residual;     // final ||b - A x||
};
void solve_refined(plx_geom *g, const RefineRequest &rq, const double *d_B, double *d_X, RefineResult &res);

// Columns of a refinement in slots [cap][2][n]: right-hand sides B, solutions X
// and FP64 residuals R, with per-slot bookkeeping.  attach() works on arrays the
// caller owns (one solve of C columns); own() + grow() keep them in the state
// (continuous batching: columns come and go between outer steps).
struct RefineState {
    struct Slot {
        enum State { FREE = 0, ACTIVE = 1, FINISHED = 2 } state = FREE;
        int32_t freq = 0, pol = 0;
        double tol = 0.0;               // absolute
        int32_t status = PLX_ERR_NOT_CONVERGED;
        int32_t outer = 0, inner_steps = 0;
        double residual = 0.0;
        int64_t tag = -1;               // request of a continuous batch
    };
    plx_geom *g = nullptr;
    RefineRequest rq;
    int cap = 0;
    const double *B = nullptr;
    double *X = nullptr;
    DevArray<double> R, ownB, ownX;
    // scratch of an outer step, cap columns
    DevArray<double> Ba, Da, AXa, nrm, Dacc, Bc, Wc;
    DevArray<int32_t> d_idx, d_fa, d_sub, d_fsub;
    std::vector<Slot> slots;
    void attach(plx_geom *geom, const RefineRequest &settings, int n_slots, const double *d_B, double *d_X);
    void own(plx_geom *geom, const RefineRequest &settings);
    int grow(int need);
    // residual norms of the ACTIVE slots: converged, non-finite or out of outer
    // steps become FINISHED with their status
    void update_status();

  private:
    void scratch(int n_cols);
};

// One outer refinement step over a state's ACTIVE slots: begin() (false when
// none is active), then while advance(&need): the caller computes the inner
// operator product `need` and calls product_done(); advance() returning false
// means the step (inner cycles, x += d, FP64 residual) is complete.
class OuterStep {
  public:
    explicit OuterStep(RefineState &s);
    ~OuterStep();
    bool begin();
    bool advance(OpInput *need);
    void product_done();

  private:
    RefineState &s_;
    std::vector<int32_t> act_, fa_, cur_;
    std::vector<double> tol_k_;
    GmresRequest in_, rin_;
    GmresResult ir_;
    std::unique_ptr<GmresStepper> run_;
    const double *bc_ = nullptr;
    int cyc_ = 0;
    bool done_ = true;
};
// One outer step of several states (geometries sharing a context) whose inner
// Arnoldi steps share one grouped operator application per step.
void refine_group_step(const std::vector<RefineState *> &states);

// analysis.cu: induced field (3 complex per point) and density (1 complex per
// point) of one solution x (complex interleaved, n_var) at P points [3][P] bohr
void field_at_points(plx_geom *g, int pol, const double *d_x, int P, const double *d_pts, double *d_field,
                     double *d_dens);

void bem_field_at_points(plx_ctx *ctx, int n, const double *centres, const double *q, double e0, int pol, int P,
                         const double *points, double *field_out);

// neighbours.cu: neighbour counts per atom (cell list on the device)
void neighbour_counts(plx_ctx *ctx, int n, int nt, const double *coord_ang, const int32_t *atom_type,
                      const int32_t *type_z, const double *r0, int32_t *nb_out, int32_t *n_nb_out);

// cholesky.cu: dense FP64 Cholesky of an n x n column-major SPD matrix (lower
// triangle) in place; returns 0 or the 1-based column of a non-positive pivot;
// and the solves L L^T X = B for nrhs columns in place
int cholesky_factor(plx_ctx *ctx, int n, double *A);
void cholesky_solve(plx_ctx *ctx, int n, const double *L, int nrhs, double *B);

// static_fq.cu: static FQ / FQFMu solves and the principal-axis rotation
int64_t static_n_var(const plx_static_desc *d);
void static_solve(plx_ctx *ctx, const plx_static_desc *d, int what, double *variables, double *energy,
                  double *polar);
void principal_axes(int n, const int32_t *z, double *coord, double *eigenvalues, double *axes);

// observables.cu
void polar_batch(plx_geom *g, int count, const int32_t *d_pol, const double *X,
                 Cplx *d_polar /* [count][3] : alpha(a, pol_c) */);

// Brackets a section with profiling events when profiling is enabled.
// Categories: 0 tensor-core T contraction, 1 FP64 T contraction, 2 Arnoldi
// orthogonalisation, 3 conductance / diagonal rows, 4 least squares and updates.
enum ProfCat { PROF_TC = 0, PROF_FP64 = 1, PROF_ORTHO = 2, PROF_ROWS = 3, PROF_LSQ = 4 };
void prof_begin(plx_ctx *ctx);
void prof_end(plx_ctx *ctx, int cat, double flops, double bytes);

// Runs fn once per (key, device) in the process; thread-safe.  Kernel attributes
// (cudaFuncSetAttribute) belong to the device that is current, and several host
// threads (one context each) may reach the same launch site.
template <typename F>
void once_per_device(const void *key, int device, F fn) {
    static std::mutex m;
    static std::set<std::pair<const void *, int>> done;
    std::lock_guard<std::mutex> lk(m);
    if (done.count({key, device})) return;
    fn();
    done.insert({key, device});
}

inline int n_blocks(int64_t work, int per_block) {
    int64_t b = (work + per_block - 1) / per_block;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace plx

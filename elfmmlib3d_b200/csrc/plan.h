// plan.h -- host orchestration of one elastostatic layer-potential evaluation.
#pragma once
#include <vector>
#include <functional>
#include <utility>
#include "devbuf.h"
#include "tree.h"
#include "fmm.h"
#include "kernels.h"
#include "rotations.h"
#include "tune.h"

namespace efmm {

// iprec -> tolerance and leaf capacity (src/elfmm3dtria.f:702-722; the ITER
// routines double the leaf capacity, src/elhfmm3dtria_iter.f:1481-1491).
double iprec_eps(int iprec);
int iprec_nbox(int iprec, int nsrc, int ntarg, bool iter);

struct OpPool {
  int p = -1;
  double eps = -1;
  DevBuf<double> mats;
  // Mixed-precision form: operators in the normalised basis (multipole
  // coefficients x w, local coefficients / w, w(n,m) = sqrt((n+m)!(n-m)!)),
  // where regular and irregular harmonics are O(1) and FP32 neither
  // overflows nor underflows; made on first use.
  DevBuf<float> mats_f;
  DevBuf<double> wnorm;   // w per real row (2 ncoef(p))
  DevBuf<int> kinds;      // operator kind per group (0 M2L, 1 M2M, 2 L2L)
  std::vector<OpDesc> descs;
  DevBuf<int> m2lg_dev;  // m2l_group on the device
  // factored form (rotation, shift along z, rotation back) of every group,
  // FP64 factorial basis and FP32 normalised basis; made on first use
  bool rot_ready = false;
  DevBuf<RotOp> rot_ops;
  DevBuf<double> rot_d;
  DevBuf<float> rot_f;
  // the FP32 factored operators as tensor-core tiles (orders <= 31); made on
  // the first FP32 pass that uses them
  bool rot_tc_ready = false;
  DevBuf<RotTcOp> rot_tc_ops;
  DevBuf<float> rot_tc_tiles;
  // the FP32 factored operators in the parity-split form (rotations as Rz
  // then Ry, re / im blocks); made on the first FP32 pass that uses them
  bool rots_ready = false;
  DevBuf<RotSOp> rots_ops;
  DevBuf<float> rots_f;
  DevBuf<long long> off;
  DevBuf<int> dim;
  int m2l_group[343];
  int m2m_group[8], l2l_group[8];
  std::vector<int> dims;
  // M2L operators of the half-space kernel U (kind 3), offsets with a
  // non-negative z component only (targets above the image sources); made
  // on first use, dense
  bool u_ready = false;
  DevBuf<double> umats;
  DevBuf<float> umats_f;
  DevBuf<long long> uoff;
  DevBuf<int> udim, ukinds, m2lug_dev;
  std::vector<int> udims;
  std::vector<OpDesc> udescs;  // the U groups (offsets, orders)
  int m2lu_group[343];
  // the U-kernel M2L in the parity-split form (FP32), made on first use
  bool us_ready = false;
  DevBuf<USOp> us_ops;
  DevBuf<float> us_pool;
};

struct Timings {  // milliseconds of the last evaluate(), CUDA events
  float total = 0, p2m = 0, m2m = 0, m2l = 0, l2l = 0, l2t = 0, near = 0, prep = 0;
  // last set_geometry(), host wall clock: tree, lists, work lists (+ gathers), operators
  float geo_tree = 0, geo_lists = 0, geo_work = 0, geo_ops = 0;
};

// Translation schedule of one kind (M2M, M2L or L2L): pairs sorted by
// operator group, one segment per (level, group); tasks are cut for a given
// number of columns per box C and cached.
struct TransSeg {
  int group, pair0, npair;
};
struct TransSched {
  DevBuf<TransPair> pairs;
  std::vector<TransSeg> segs;
  std::vector<std::pair<int, int>> lev;  // segment ranges in execution order
  int C = -1;
  const void* pool = nullptr;  // operator pool the tasks were cut for
  DevBuf<TransTask> tasks;
  std::vector<std::pair<int, int>> lev_tasks;  // task ranges in execution order
  // column tiles of the factored kernel (cut for C, tile width and pool)
  int rC = -1, rW = -1;
  const void* rpool = nullptr;
  DevBuf<TransTask> rtasks;
  std::vector<std::pair<int, int>> lev_rtasks;  // task ranges in execution order,
  std::vector<int> lev_rdim;                     // each with its largest operator size
  // tensor-core form: segments, 32-column tasks, and per launch (a level,
  // or all levels of an M2L stage) the task range and its largest order
  int tcC = -1;
  const void* tcpool = nullptr;
  DevBuf<RotTcSeg> tcsegs;
  DevBuf<RotTcTask> tctasks;
  struct TcBatch {
    int task0, ntask, pmax;
  };
  std::vector<TcBatch> tcb;
  // tiles of the parity-split U-kernel M2L (run_u_split), cut for uC
  int uC = -1, untask = 0;
  const void* upool = nullptr;
  DevBuf<TransTask> utasks;
  void clear() {
    segs.clear();
    lev.clear();
    C = -1;
    pool = rpool = nullptr;
    lev_tasks.clear();
    rC = rW = -1;
    lev_rtasks.clear();
    lev_rdim.clear();
    tcC = -1;
    tcpool = nullptr;
    tcb.clear();
    uC = -1;
    upool = nullptr;
  }
};

// Waves of leaves for the two-stage P2M / L2T products: per wave the leaf
// range, its product tasks and scratch extent, uploaded once per key (kind,
// column count, element type) and reused by every later pass.
struct WaveSet {
  struct Wave {
    int nwl;
    long long wl0;
    int ntask;
    long long t0;
    int maxn;
    long long used, nodes;
  };
  long long key = -1;
  // resident: one wave whose geometry-only features (unit multipoles, L2T
  // functionals) stay in the scratch between passes; feat_valid: computed
  bool resident = false, feat_valid = false;
  // split: the resident wave keeps its geometry-only operand as split tiles
  // and runs k_tc_bulk (btasks; off3 the other operand's split tiles)
  bool split = false;
  DevBuf<BulkTask> btasks;
  double bulk_flops = 0;  // useful flops of btasks
  std::vector<Wave> w;
  std::vector<GemmTask> htasks;
  DevBuf<int> leaves;
  DevBuf<long long> off1, off2, off3;
  DevBuf<GemmTask> tasks;
  void clear() {
    key = -1;
    resident = feat_valid = split = false;
    w.clear();
    htasks.clear();
  }
  void upload(const std::vector<int>& wl, const std::vector<long long>& o1, const std::vector<long long>& o2,
              const std::vector<long long>& o3, const std::vector<GemmTask>& t, cudaStream_t st);
};

class Plan {
 public:
  Plan(int device, cudaStream_t stream);
  ~Plan();
  // geometry in user order, device pointers: tri (n,3,3), nrm (n,3), src (n,3), tgt (nt,3)
  int set_geometry(int n, const double* d_tri, const double* d_nrm, const double* d_src, int nt,
                   const double* d_tgt, int iprec, bool iter, bool mindlin);
  // A forest of independent problems for the following set_geometry calls:
  // f5 = {root centre x, y, z, root side, level} as build_tree's forest (the
  // Mindlin root needs centre z = 0); null: one problem.
  // Leaf capacity of the following set_geometry calls (boxes split while
  // they hold more sources or targets); <= 0: the iprec table.
  void set_leaf(int nbox) { leaf_override_ = nbox; }
  void set_forest(const double* f5) {
    forest_on_ = f5 != nullptr;
    for (int i = 0; i < 5; i++) forest_[i] = f5 ? f5[i] : 0.0;
  }
  // densities in user order (device); outputs in user order (device):
  // u_src (n,3), e_src (n,3,3), u_tgt (nt,3), e_tgt (nt,3,3); null pointers disable them.
  // mode 0: analytic near field; 1: compute and store the near-field
  // operator (ITER first call), then apply it; 2: apply the stored operator
  // (ITER later calls; same layers/outputs/Lame constants as the store,
  // else IER_HANDLE).  do_far = false skips the far field (near part only).
  int evaluate(double rlam, double rmu, const double* d_ssl, const double* d_sdl, double* d_u_src,
               double* d_e_src, double* d_u_tgt, double* d_e_tgt, int mode = 0, bool do_far = true);
  long long stored_doubles() const { return store_valid_ ? (long long)store_.size() : 0; }
  bool store_valid() const { return store_valid_; }
  // tolerance floor of the mixed form's orders (<= 0: the iprec orders)
  void set_mixed_floor(double eps);
  int mixed_order() const { return p_mixed_; }
  // R right-hand sides at once: densities (R, n, 3) user order, outputs
  // (R, n, 3) / (R, n, 3, 3) / (R, nt, 3) / (R, nt, 3, 3) user order.  The
  // tree, lists and operators are shared; the near-field pair responses are
  // computed once and contracted with all right-hand sides.
  // precision 0: FP64 throughout; 1: mixed (P2M products and translations
  // in FP32 with FP32 expansions, everything else FP64).  mode as in
  // evaluate: 1 stores the near-field operator (then replays it for all
  // right-hand sides), 2 replays a stored one.
  int evaluate_batch(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                     double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt,
                     int precision = 0, int mode = 0);
  // Half-space image part (Mindlin) of the layer potentials on triangles in
  // z <= 0, at the original targets x (R, nt, 3) / (R, nt, 3, 3), user
  // order.  The plan's geometry must have been set with mindlin = true and
  // the REFLECTED targets (x1, x2, -x3) as its targets.  Far field: the
  // anti-image passes and the two 1/r potentials of the C piece through the
  // Laplace translations, the U potential of the B piece through its own
  // dense M2L (kind 3); near field: refined quadrature of the whole image
  // kernel over the near lists, stored and contracted with all right-hand
  // sides.  precision and mode as in evaluate_batch (mode 0 computes the
  // near-field blocks for this call only).
  int evaluate_image(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                     double* d_u_tgt, double* d_e_tgt, int precision = 0, int mode = 0);
  // The same calls replayed as one CUDA graph: the first call with a new
  // key (parameters and device pointers) runs the pass, captures a second
  // identical pass and launches the graph; later calls with the same key
  // only launch it.  Batch: mode 0 or 2 (the store made by an earlier mode-1
  // call); image: mode 2.  New data must be written into the same buffers.
  int evaluate_batch_graph(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                           double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, int precision,
                           int mode);
  int evaluate_image_graph(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                           double* d_u_tgt, double* d_e_tgt, int precision);
  // useful flops per expansion column of one pass: P2M, M2M, M2L, L2L, L2T
  void flops_per_column(double* f5) const;
  // Flops of one pass's translation launches for R right-hand sides at the
  // orders of the given form (mixed: the mixed form's orders and pool):
  // f3 = M2M, M2L, L2L (factored form: two rotations and the z shift per
  // pair and column; dense: 2 dim^2); image: the image plan's schedules
  // (6R Laplace columns, R columns of U with its dense M2L).
  void translation_flops(int R, bool mixed, double* f3);
  // all-pairs direct sum on the same geometry (no tree needed)
  // nsub > 0: only the first nsub source points (centroids), no targets
  int evaluate_direct(double rlam, double rmu, const double* d_ssl, const double* d_sdl,
                      double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, int nsub = 0);
  cudaStream_t stream() const { return st_; }
  const Tree& tree() const { return tr_; }
  Timings timings;
  int n() const { return n_; }
  bool points() const { return points_; }
  int nt() const { return nt_; }
  int order() const { return p_; }
  int nbox() const { return nbox_; }
  long long near_pairs() const { return near_pairs_; }
  long long m2l_pairs() const { return (long long)m2l_pairs_h_; }
  int kernel_launches() const { return launches_; }
  // P2M product stage of the last evaluate_batch / evaluate_image: device ms
  // (CUDA events around each product launch) and useful flops
  double product_ms() const { return product_ms_; }
  void near_stats(double* out) const;
  double product_flops() const { return product_flops_; }
  bool far_enabled() const { return far_; }

 private:
  void build_worklists();
  int batch_pass(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                 double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, bool mixed, int mode);
  int store_alloc(int flags, double rlam, double rmu);
  int image_pass(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl, double* d_u_tgt,
                 double* d_e_tgt, bool mixed, bool store_now);
  void ensure_uops();
  void ensure_mats_f();
  int build_image_sched();
  void build_chunks(int do_src, int do_tgt);
  bool mindlin_ = false, img_sched_ = false;
  bool forest_on_ = false;
  // keep the geometry-only features of the two-stage P2M / L2T between
  // passes when they fit (store / replay and graph passes)
  bool resident_ = false, graph_pass_ = false;
  bool resident_fits(long long elems, size_t esz, size_t cap_bytes);
  // the resident L2T wave from split operands (mixed form): layout of the
  // per-leaf split functionals, split local expansions and products for P
  // points per leaf and C columns; false when it does not fit
  bool l2t_split_layout(WaveSet& W, int D, int C, const std::vector<int>& P, long long key);
  void l2t_split_run(const L2TArgs& la, int R, const float* local, bool image);
  bool p2m_split_layout(WaveSet& W, int D, int R, int nk, int ns, bool image, long long key);
  void bulk_timed(int ntask, double flops, const BulkTask* dtasks, const float* A, const float* B, float* C, int bn);
  int leaf_override_ = 0;
  double forest_[5] = {0, 0, 0, 0, 0};
  TransSched m2lv_img_, m2lu_, l2l_img_, l2l_img_u_, m2m_u_;
  template <class T>
  void p2m_img_twostage(const P2MArgs& pa, int R, T* mpole);
  void l2t_img_twostage(const L2TArgs& la, int R, const double* local, const float* local_f);
  template <class T>
  void run_dense(TransSched& S, int C, const T* mats, const T* src, T* dst);
  DevBuf<double> img_mp_, img_lc_;
  // event pairs around the P2M product launches of one pass
  std::vector<cudaEvent_t> pev_;
  int npev_ = 0;
  double product_ms_ = 0, product_flops_ = 0;
  void product_begin();
  void product_end();
  void product_collect();
  template <class T>
  void product_timed(int ntask, const std::vector<GemmTask>& tasks, long long t0, const GemmTask* dtasks, const T* F,
                     const T* W, T* C, int bn = 128);
  WaveSet p2m_waves_, l2t_waves_;
  bool capturing_ = false;
  int rc_last_ = 64;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
  std::vector<double> gkey_;
  long long graph_launches_ = 0;
  void rec(int i);
  void graph_reset();
  int run_graph(const std::vector<double>& key, const std::function<int()>& pass);
  DevBuf<float> img_mp_f_, img_lc_f_;
  DevBuf<float> mpole_f_, local_f_;
  DevBuf<int> chunk_leaf_, chunk_e0_;  // (near leaf, first point) per batched near-field CTA
  int nchunk_ = 0, chunk_key_ = -1;
  std::vector<int> l2t_sc_h_, l2t_tc_h_;  // per L2T leaf
  std::vector<int> l2t_h_;                // L2T leaves
  DevBuf<double> l2t_scratch_;            // functionals + sums of one wave of leaves
  void l2t_twostage(const L2TArgs& la, int R, int do_src, int do_tgt, bool mixed = false);
  std::vector<int> p2m_h_, p2m_sc_h_;     // P2M leaves and their triangle counts
  DevBuf<double> p2m_scratch_;            // node features + weights of one wave of leaves
  DevBuf<int> wave_leaves_;
  DevBuf<long long> wave_foff_, wave_woff_, wave_noff_;
  DevBuf<double> wave_nrec_;
  DevBuf<GemmTask> wave_tasks_;
  template <class T>
  void p2m_twostage(const P2MArgs& pa, int R, T* mpole);
  // P2M through unit-density multipoles (free-space 4 kinds, or the image
  // plan's 7); false when the order is too high for its kernel
  template <class T>
  bool p2m_factored(const P2MArgs& pa, int R, T* mpole, bool image);
  DevBuf<int> lchunk_leaf_, lchunk_e0_;   // (L2T leaf index, first point) per product-form L2T CTA
  int nlchunk_ = 0, lchunk_key_ = -1;
  void ensure_ops();
  int dev_;
  cudaStream_t st_;
  int n_ = 0, nt_ = 0, iprec_ = 2, nbox_ = 40, p_ = 0;
  double eps_ = 0.5e-6;
  // Mixed form (precision 1): expansion and translation orders for
  // max(eps_, mixed_floor_) -- no truncation finer than the FP32 rounding
  // of the result; mixed_floor_ <= 0 keeps the iprec orders.
  double mixed_floor_ = 0.5e-7, eps_mixed_ = 0.5e-6;
  int p_mixed_ = 0;
  friend struct MixedOrders;
  bool far_ = false;
  Tree tr_;
  DevBuf<double> tri_s_, nrm_s_, src_s_, tgt_s_;
  DevBuf<double> tri_u_;  // user-order triangles (for the direct sum)
  DevBuf<double> src_u_, tgt_u_;
  DevBuf<int> p2m_leaves_, l2t_leaves_, near_leaves_, near_start_, near_items_;
  int np2m_ = 0, nl2t_ = 0, nnear_ = 0;
  std::vector<int> near_sc_h_, near_tc_h_, near_ntri_h_;  // per near leaf
  DevBuf<int> near_ntri_;
  DevBuf<long long> near_base_;
  std::vector<long long> near_base_h_;
  // FP32 product-layout copy of the stored near field for mixed replays on
  // the tensor cores (built from store generation store_tc_gen_), the
  // per-leaf product tasks and the density / product scratch
  DevBuf<float> store_f_, ntc_scratch_;
  // the FP32 copy's per-leaf offsets (16-byte aligned, rows padded to a
  // multiple of 4 floats, so that its tiles copy with 16-byte cp.async)
  std::vector<long long> fbase_h_;
  DevBuf<long long> fbase_;
  DevBuf<double> ntc_cbuf_;
  DevBuf<long long> ntc_soff_, ntc_coff_;
  DevBuf<GemmTask> ntc_tasks_;
  long long store_gen_ = 0, store_tc_gen_ = -1, ntc_key_ = -1, ntc_stot_ = 0, ntc_ctot_ = 0;
  int ntc_ntask_ = 0;
  // the pre-split store (tiles of 128 rows x 32 k, TF32 head then tail; the
  // bulk-copy product of tc_bulk.cu), used instead of store_f_ when it
  // fits: per-leaf tile bases and K tiles, the product tasks
  bool near_split_ = false;
  int near_req_ = -1;  // split_variant() when the copy was made
  DevBuf<float> store_s_;
  std::vector<long long> tbase_h_;
  std::vector<int> nkt_h_;
  DevBuf<long long> tbase_;
  DevBuf<BulkTask> nsp_tasks_;
  // events around the split near-field product (outside graph capture)
  cudaEvent_t nev_[2] = {nullptr, nullptr};
  bool near_timed_ = false;
  double near_bytes_ = 0;
  bool near_tc_ready(const NearArgs& na);
  void near_tc(const NearArgs& na, int R, const double* g0, const double* g1, int n, int nt);
  DevBuf<double> store_;
  bool store_valid_ = false;
  int store_flags_ = 0, store_K_ = 0;
  double store_lam_ = 0, store_mu_ = 0;
  long long near_pairs_ = 0;
  TransSched m2m_, m2l_, l2l_;
  void cut_tasks(TransSched& S, int C, const std::vector<int>* dims = nullptr);
  void cut_rot_tasks(TransSched& S, int C, int W);
  void ensure_factored(bool tc = false);
  void ensure_split();
  // the U-kernel M2L in the parity-split form (mixed form; ELFMM3D_USPLIT=0:
  // the dense FP32 operators)
  void ensure_usplit();
  bool usplit_on() const;
  void run_u_split(int C, const float* src, float* dst);
  // whether the FP32 translations run in the parity-split form
  bool split_rot() const;
  // the FP32 translations of a schedule on the tensor cores (rot_tc.cu)
  bool rot_tc_usable() const;
  void cut_tc_tasks(TransSched& S, int C, bool one_launch);
  void run_translations_tc(TransSched& S, int C, const float* src, float* dst, bool one_launch);
  // autotuned engine of the FP32 translations per stage (M2M, M2L, L2L):
  // 0 tensor cores, 1 CUDA cores; chosen at the start of a mixed pass
  // (tune_begin), reported with the stage times at its end (tune_end)
  int trans_cand_[3] = {0, 0, 0};
  TuneKey trans_key_[3];
  bool trans_tuning_ = false;
  void tune_begin(int kind, int C);
  void tune_end();
  // A pass of the other precision than the last one releases the large
  // buffers only the last one's form uses (FP32 expansions, the FP32 copy
  // of the stored near field and the tensor-core intermediates; or the FP64
  // expansions of many right-hand sides), so that the memory a form finds,
  // and with it the size of its waves and right-hand-side chunks, does not
  // depend on which form ran before.  Captured graphs are dropped with them.
  int last_mixed_ = -1;
  void switch_precision(bool mixed);
  // particles (set_geometry with no triangles): sources are points, nrm the
  // dipole orientations; the FP64 single-right-hand-side forms only
  bool points_ = false;
  DevBuf<double> nu_u_;  // dipole orientations, user order (direct sum)
  bool factored_ = true;  // translations in factored form when they fit
  bool p2m_unit_ = true;  // batched P2M through unit-density multipoles (else node products)
  template <class T>
  void run_translations(TransSched& S, int C, const T* mats, const T* src, T* dst);
  size_t m2l_pairs_h_ = 0;
  DevBuf<int> m2l_cnt_, m2l_cursor_;
  DevBuf<double> mpole_, local_;
  DevBuf<double> ssl_s_, sdl_s_, u_s_, e_s_, ut_s_, et_s_;
  DevBuf<TriRec> trir_;
  OpPool* ops_ = nullptr;
  cudaEvent_t ev_[10];
  int launches_ = 0;
};

}  // namespace efmm

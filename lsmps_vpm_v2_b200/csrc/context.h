// The context behind `vpm_ctx`: device, stream, one device arena per
// dimension, timing events and the state of the last evaluation.
#pragma once

#include <string>
#include <vector>

#include "fmm2d.cuh"
#include "fmm3d.cuh"

namespace vpm {

struct Selector;  // learned (caps, p) selector state (selector.cu)
void drop_selector(Selector* s);

// Stage marks of one evaluation: 0 start, 1 keys+sort, 2 tree levels,
// 3 lists, 4 P2M+M2M, 5 M2L, 6 L2L, 7 M2P+L2P, 8 P2P (end).
constexpr int kStageEvents = 9;

// Output mode of a 2D evaluation (the `velocity` argument below): 0 field
// (Ex, Ey), 1 velocity (u, v), kModePotential the potential (one output).
constexpr int kModePotential = 2;

struct Caps3D {
    int n = 0, cells = 0;
};

struct Caps2D {
    int n = 0, cells = 0, P = 0;
    long long l1 = 0, l3 = 0;
};

// Host copy of a 2D tree for the parity dumps.
struct HostTree2D {
    int nc = 0, nl = 0, n = 0;
    std::vector<int32_t> lo, hi, src, ix, iy, leafidx, leaf_cells, l2, l4, l1, l3;
    std::vector<uint8_t> flags, level, l2n, l4n;
    std::vector<double> cx, cy;
    std::vector<uint32_t> perm, l1off, l3off;
    std::vector<int64_t> id;
    std::vector<int> by_id;
};

// Size of the mixed-precision work area inside the 2D arena.
size_t mixed_bytes(int n, int cap_cells, int P);

struct Ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // Second stream of a captured evaluation: lists 1/3 and the near field run
    // on it while the main stream builds lists 2/4 and the far field.
    cudaStream_t side = nullptr;
    cudaStream_t side2 = nullptr;   // lists 2/4 while the main stream runs P2M + M2M
    cudaEvent_t fork2 = nullptr, join2 = nullptr, join3 = nullptr;
    cudaEvent_t ev_up = nullptr, ev_l13 = nullptr, join4 = nullptr;   // upward done, lists 1/3 done, M2P done
    cudaStream_t side3 = nullptr;   // CSR of lists 1/3 while the near field runs from the slots
    cudaEvent_t ev_slots = nullptr, join5 = nullptr;   // list slots done, near field of spilled leaves done
    // moments of all but the M2M loop's cells done; M2L of the parents below them done
    cudaEvent_t ev_small = nullptr, ev_m2ld = nullptr;
    // Host entry points: the strengths (or vorticity and core size) are
    // copied on `upload` while the main stream sorts the particles and builds
    // the tree and lists; `q_ready` (recorded on `upload`) is set while an
    // evaluation waits for them, and `ev_qg` marks the strengths in tree order.
    cudaStream_t upload = nullptr;
    cudaEvent_t ev_upload = nullptr, ev_q = nullptr, ev_qg = nullptr;
    cudaEvent_t q_ready = nullptr;
    double *near_x = nullptr, *near_y = nullptr;
    std::string last_error;
    unsigned* d_err = nullptr;
    cudaEvent_t ev[kStageEvents] = {};

    // 2D arena
    void* arena2d = nullptr;
    size_t arena2d_bytes = 0;
    Caps2D cap;
    bool grow = false;
    double *in_x = nullptr, *in_y = nullptr, *in_q = nullptr, *out0 = nullptr, *out1 = nullptr;
    uint8_t* in_act = nullptr;
    Tree2D tree{};
    TreeScratch2D ts{};
    Lists2D lists{};
    Expansions2D ex2{};
    void* mixed_base = nullptr;
    float* tc_rows = nullptr;   // tensor-core M2L: scaled TF32 multipole rows
    float* tc_ops = nullptr;    //                  list-2 operators (hi, lo)
    int coef_P = -1, coef_binom = -1;

    // CUDA graph of the device entry point (capture once, replay)
    struct GraphKey {
        const void* ptr[6];
        int n, K, velocity;
        double uinf, vinf;
        vpm_fmm_params p;
        cudaStream_t stream;
        void* arena;
        int deferred;   // the strengths arrive on `upload` (q_ready)
    };
    cudaGraphExec_t gexec = nullptr;
    GraphKey gkey{};
    bool capturing = false;      // a CUDA graph capture is open on `stream`
    bool split_capture = false;  // ... one graph per stage (use_graph = 2)
    bool last_timed = false;     // the stage events of the last evaluation are valid
    cudaGraphExec_t stage_exec[kStageEvents - 1] = {};
    // Ring of stage-event sets: with the ring on, each timed evaluation records
    // into the next slot, so many evaluations can run back to back and be
    // read afterwards (vpm_stage_history).
    static constexpr int kRing = 64;
    cudaEvent_t ring[kRing][kStageEvents] = {};
    int ring_on = 0, ring_head = 0, ring_count = 0, ring_cur = -1;
    bool last_was_graph = false;
    int graph_launches = 0;

    // 3D arena
    void* arena3d = nullptr;
    Caps3D cap3;
    double* in3[7] = {};          // x, y, z, alpha_x, alpha_y, alpha_z (or vorticity), s
    uint8_t* in3_act = nullptr;
    double* out3[3] = {};
    Tree3D tree3{};
    Scratch3D s3{};
    double* bbox3 = nullptr;
    bool have_tree3 = false;
    bool last_treecell3 = false;   // the last 3D build was a TreeCell
    uint8_t* in3_tgt = nullptr;
    int last_n3 = 0;
    float last_ms3 = 0.f;
    int last_launches3 = 0;

    Selector* selector = nullptr;

    // particles per block of the cooperative sort (keys_sort2d; at most one
    // block per SM): 1024 for a solve with the GPU to itself (the 65,536-
    // particle lattice spreads over 64 SMs: 0.183 -> 0.179 ms against 2048),
    // more in the sub-contexts of a batch, whose solves share the GPU
    int sort_items = 1024;
    // mixed form: the M2L of the levels below the large cells beside their M2M
    // loop (one graph per solve); off in the sub-contexts of a batch, whose
    // small solves share the GPU and gain nothing from the extra launch
    bool split_m2l = true;

    // batched solves (batch2d.cu)
    std::vector<Ctx*> subs;
    std::vector<cudaEvent_t> join_ev;
    cudaEvent_t fork_ev = nullptr;
    cudaGraphExec_t batch_exec = nullptr;
    std::vector<int64_t> batch_key;
    int batch_subs = 0;
    int batch_streams = 0;                       // streams of the tuned batch graph
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};  // timing of the stream-count tuning
    void* batch_in = nullptr;
    size_t batch_in_bytes = 0;

    // last evaluation
    bool have_tree = false;
    int last_n = 0;
    int last_launches = 0;
    int depth_retry = 0;
    vpm_fmm_params last_params{};
    HostTree2D host_tree;

    ~Ctx();
    int init(int dev);
    int fail(int status, const std::string& msg);
    int fail_cuda(cudaError_t e, const char* what);
    int map_err(unsigned bits);
    int check_params(const vpm_fmm_params* prm, vpm_fmm_params& out);
    int plan_caps(int n, const vpm_fmm_params& p, int& cells, long long& l1, long long& l3);
    int reserve2d(int n, int cap_cells, int P, long long cap_l1, long long cap_l3);
    int enqueue2d(const double* x, const double* y, const double* q, const uint8_t* act, int n,
                  const vpm_fmm_params& p, int K, double* o0, double* o1, int velocity, double uinf, double vinf,
                  bool tree_only);
    int run2d_host(const double* x, const double* y, const double* q_or_omega, const double* s, const uint8_t* act,
                   int64_t n, const vpm_fmm_params* prm, double* o0, double* o1, int velocity, double uinf,
                   double vinf, vpm_fmm_stats* stats, bool tree_only);
    int collect_stats(vpm_fmm_stats* s);
    int count_interactions(vpm_fmm_stats* s);
    int fetch_tree(HostTree2D& h);
    int ensure_coefs(const vpm_fmm_params& p);
    int enqueue_m2l(const vpm_fmm_params& p, cudaStream_t st, int* launches);
    int launch2d(const double* x, const double* y, const double* q, const uint8_t* act, int n,
                 const vpm_fmm_params& p, int K, double* o0, double* o1, int velocity, double uinf, double vinf);
    int reserve3d(int n, int cap_cells);
    // treecell: the 3D TreeCell path instead of the octree; target (device,
    // caller order, may be null): evaluate only flagged particles.
    int enqueue3d(const double* x, const double* y, const double* z, const double* ax, const double* ay,
                  const double* az, const uint8_t* act, int n, const vpm_fmm_params& p, double* u, double* v,
                  double* w, double uinf, double vinf, double winf, bool tree_only, bool treecell,
                  const uint8_t* target);
    int run3d_host(const double* x, const double* y, const double* z, const double* a0, const double* a1,
                   const double* a2, const double* s, const uint8_t* act, int64_t n, const vpm_fmm_params* prm,
                   double* u, double* v, double* w, double uinf, double vinf, double winf, vpm_fmm_stats* stats,
                   bool tree_only, bool treecell, const uint8_t* target);
    int batch2d(int ns, const int64_t* offs, const double* x, const double* y, const double* q, const uint8_t* act,
                const vpm_fmm_params& p, double* ex, double* ey);
    int batch_errors(unsigned* bits);
    int prepare_batch(int ns, const int64_t* offs, const vpm_fmm_params& p, int S, const std::vector<int>& stream_of);
    int enqueue_batch(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                      const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey, int S,
                      const std::vector<int>& stream_of, const std::vector<int>& order);
    int capture_batch(int ns, const int64_t* offs, const double* x, const double* y, const double* q,
                      const uint8_t* act, const vpm_fmm_params& p, double* ex, double* ey, int S,
                      cudaGraphExec_t* out);
    void drop_batch();
    void drop_graph();
    void begin_ring();
    void end_ring();
    int record(int i);
};

// FP32 P2P of the mixed form (packed FP32x2, warp per leaf); near_only: the
// near field alone in tree order into out0/out1. lists: where list 1 comes
// from: the CSR (kP2PListCsr), the fixed slots of the one-pass list build
// (kP2PListSlots: leaves whose list outgrew them are skipped) or, for exactly
// those leaves, the CSR (kP2PListSpill). Every leaf sums its sources in the
// same order whichever source is used.
cudaError_t fmm2d_p2p_f32(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* out0, double* out1,
                          int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st, int* launches,
                          bool near_only = false, int lists = kP2PListCsr);
// FP64 P2P on an AoS copy of the particles (`aos`, n entries); kernel choice as
// for fmm2d_p2p_f32.
cudaError_t fmm2d_p2p_f64_tma(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double4* aos, double* out0,
                              double* out1, int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st,
                              int* launches, int max_par, bool near_only = false);
// Far field (M2P + L2P) plus the near field nx/ny (tree order), written in the
// caller's order (field or velocity). With m2p_done the list-3 sums are
// already in e.fx/e.fy (fmm2d_m2p) and only L2P is added (same result).
cudaError_t fmm2d_eval_combine(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, const double* nx,
                               const double* ny, double* out0, double* out1, int velocity, double u_inf, double v_inf,
                               unsigned* err, cudaStream_t st, int* launches, bool m2p_done = false);
// M2P over list 3 of every leaf's particles into e.fx/e.fy (tree order);
// lists: where list 3 comes from, as for fmm2d_p2p_f32 (the slots pass skips
// the leaves whose list outgrew them, the spill pass takes exactly those).
cudaError_t fmm2d_m2p(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches, int lists = kP2PListCsr);
cudaError_t fmm2d_p2p_out(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* out0, double* out1,
                          int velocity, double u_inf, double v_inf, unsigned* err, cudaStream_t st, int* launches);

}  // namespace vpm

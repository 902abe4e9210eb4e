// exg_internal.h -- host-side context of the B200 MPM step and the kernel
// launchers shared by the translation units of libexg.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <string>
#include <vector>
#include "exg_common.cuh"

namespace exg {

// NVTX range over a scope (the counterpart of the reference's BL_PROFILE
// regions, e.g. MPMParticleContainer::updateVolume in
// mpm_particle_timestep.cpp:133): the entry points and the stages of a step
// show up by name in Nsight timelines.  Header-only NVTX3: without a
// profiler attached each push/pop is a no-op call.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define EXG_RANGE(name) ::exg::NvtxRange exg_nvtx_range_(name)

enum P2GFlags { PF_MASS = 1, PF_VEL = 2, PF_FORCE = 4, PF_TEMP = 8, PF_SRC = 16 };
// Nodal kernel modes.
enum NodeMode {
    NM_MERGE = 0,      // merge P2G partials into the dense arrays + normalise (P2G_Momentum)
    NM_FUSED = 1,      // merge + backup + time update + BCs + store delta (one USL step)
    NM_MUSL2 = 2,      // merge momentum, normalise with the stored mass, BCs, store delta (MUSL pass 2)
};
// Thermal nodal operations (launch_temp_node_op).
enum TempNodeOp {
    TN_BACKUP = 0,     // backup_current_temperature
    TN_TIME_UPDATE = 1,  // Nodal_Time_Update_Temperature
    TN_DELTA = 2,      // store_delta_temperature
};
// walls_mask of launch_temp_bcs
enum TempWalls {
    TW_OFF = 0,        // no domain-wall pass
    TW_ON = 1,         // wall pass reading the stored temperatures
    TW_MASKED = 2,     // wall pass in a fused step: nodes below the mass tolerance read as 0
};
// Fused G2P modes.
enum G2PMode {
    GM_FULL = 0,       // G2P vel + strain rate + F, move, volume, stress, reductions (USL)
    GM_VEL = 1,        // G2P vel only (MUSL pass 1)
    GM_STRAIN = 2,     // G2P strain rate + F, move, volume, stress, reductions (MUSL pass 2)
};

struct SortBufs {
    uint32_t *key = nullptr;
    int32_t *perm = nullptr;
    int32_t *bucket = nullptr;
    int *tile_count = nullptr;   // [ntiles]
    int *tile_fill = nullptr;    // [ntiles]
    int *tile_start = nullptr;   // [ntiles]
    int *active = nullptr;       // [ntiles] active tile ids (ascending)
    int *slot = nullptr;         // [ntiles] index in active list or -1
    int *touched = nullptr;      // [ntiles] tiles whose nodes the nodal kernel writes
    long long *touched_step = nullptr;  // [ntiles] last step the tile was touched
    int *cell_start = nullptr;   // [ntiles][T^3 + 1] per-cell particle ranges of each non-empty tile
    int *item_start = nullptr;   // [ntiles + 1] first fused-G2P work item of each active tile
};

struct Ctx;
// True when the fused G2P can run its lean variant: no level-set bodies, no
// UDF walls, no temperature, total strain, linear-elastic and Tait materials
// only (exg_api.cu)
bool g2p_lean(const Ctx &c);
// positions and integer fields back to upload order (exg_kernels.cu)
void d2h_positions(Ctx &c, double *const x[3], const int32_t *pid, double *host, long long n);
void d2h_int(Ctx &c, const void *src, int bytes, const int32_t *pid, int32_t *host, long long n);

// launchers (exg_kernels.cu; _fp64/_fp32 variants come from the two
// precision builds of that file)
void upload_tables_fp64();
void upload_tables_fp32();
void launch_keys(Ctx &c);
void launch_sort_rest(Ctx &c, bool touched_list);
void launch_dt_finalize(Ctx &c, bool reset);
void launch_reset_accum(Ctx &c, unsigned long long *bounds, unsigned long long *dtmin);
void launch_scales_from(Ctx &c, const unsigned long long *bounds);
void launch_time_advance(Ctx &c);
void launch_node_reset(Ctx &c);
#define EXG_DECL_PREC(sfx)                                                      \
    void launch_state_reduce##sfx(Ctx &c, unsigned long long *bounds, unsigned long long *dtmin); \
    void launch_p2g##sfx(Ctx &c, int flags);                                     \
    void launch_nodes##sfx(Ctx &c, int mode, int flags, bool all_tiles);         \
    void launch_g2p_fused##sfx(Ctx &c, int mode);                                \
    void launch_copy_lost##sfx(Ctx &c);                                          \
    void launch_g2p_simple##sfx(Ctx &c, int uv, int us, double dt);              \
    void launch_node_backup##sfx(Ctx &c);                                        \
    void launch_node_time_update##sfx(Ctx &c, double dt);                        \
    void launch_node_bcs##sfx(Ctx &c);                                           \
    void launch_move##sfx(Ctx &c, double dt);                                    \
    void launch_volume##sfx(Ctx &c);                                             \
    void launch_stress##sfx(Ctx &c, double time, double dt, bool total = false);  \
    void launch_diag##sfx(Ctx &c, double *out_dev);                              \
    void launch_temp_node_op##sfx(Ctx &c, int op, double dt);                     \
    void launch_temp_bcs##sfx(Ctx &c, int walls_mask, int udf, int ls, int dirichlet_only); \
    void launch_g2p_temp##sfx(Ctx &c, int upd_T, int upd_q);                     \
    void launch_fill_node##sfx(Ctx &c, int comp, double value);                   \
    void h2d_field##sfx(Ctx &c, void *dst, const double *host, long long n, double sub); \
    void d2h_field##sfx(Ctx &c, const void *src, const int32_t *pid, double *host, long long n, double add);
EXG_DECL_PREC(_fp64)
EXG_DECL_PREC(_fp32)

// A batch of independent scenes (batch.cu side of exg_batch): scene
// contexts, a shared stream, the batch control block and the scene
// descriptors for both particle-buffer parities.
struct Batch {
    std::vector<Ctx *> scenes;
    cudaStream_t stream = nullptr;
    int precision = 0;
    BatchCtl *bctl = nullptr;            // device
    Ctl **ctls = nullptr;                // device: each scene's control block
    void *desc[2] = {nullptr, nullptr};  // device SceneDesc<R>[n], one array per parity
    std::vector<unsigned char> desc_host[2];
    SortDesc *sdesc[2] = {nullptr, nullptr};  // device SortDesc[n], one array per parity
    std::vector<unsigned char> sdesc_host[2];
    int total_blocks = 0, total_tiles = 0;    // of the per-particle and per-tile batched kernels
    // per-stage device timing (exg_batch_set_stage_timing): events between
    // the sort, P2G, nodal and G2P launches of eager steps
    bool timing = false;
    cudaEvent_t ev[5] = {};
    double stage_ms[5] = {};
    size_t desc_bytes = 0;
    int parity = 0;                      // flips every step
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool warm[2] = {false, false};
    int lean = -1;                       // G2P variant the graphs hold (g2p_lean of every scene)
};
// Uploads the scene descriptors of both parities; true when they changed.
bool batch_descriptors_fp64(Batch &b);
bool batch_descriptors_fp32(Batch &b);
// Batched sort and bookkeeping of every scene (one launch per kernel):
// step start (dt, accumulators, bounds), keys, tile scan, scatter, tile
// sort, touched tiles, fixed-point scales, then k_batch_plan.
void launch_batch_sort(Batch &b);
// The batched P2G, nodal and G2P launches separately (stage timing).
void launch_batch_p2g_fp64(Batch &b);
void launch_batch_p2g_fp32(Batch &b);
void launch_batch_nodes_fp64(Batch &b);
void launch_batch_nodes_fp32(Batch &b);
void launch_batch_g2p_fp64(Batch &b);
void launch_batch_g2p_fp32(Batch &b);
// Batched end of step: particles outside the domain and the time advance.
void launch_batch_finish_fp64(Batch &b);
void launch_batch_finish_fp32(Batch &b);
// k_batch_plan + batched P2G, nodal and fused G2P kernels (USL step).
void launch_batch_plan(Batch &b);
void launch_batch_core_fp64(Batch &b);
void launch_batch_core_fp32(Batch &b);

struct Ctx {
    exg_specs specs;
    Params P;
    int precision;  // EXG_PREC_*
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // particles (double buffered: a = current, b = reorder target)
    long long np = 0, cap = 0;
    void *pa = nullptr, *pb = nullptr;  // Parts<R>* host-side copies
    std::vector<void *> allocs_a, allocs_b;
    // material table
    Material *mat_dev = nullptr;
    size_t mat_cap = 0;
    std::vector<Material> mats;
    // nodes
    void *nodes = nullptr;             // Nodes<R> host copy (device pointers)
    std::vector<void *> node_allocs;
    double *ls[kMaxBodies] = {};       // nodal level sets (FP64)
    // UDF wall tables [lo/hi][dir] (FP64)
    double *udf_tab[2][3] = {};
    std::vector<double> udf_host[2][3];
    // UDF wall-temperature tables [lo/hi][dir] (FP64, two values per face node)
    double *udfT_tab[2][3] = {};
    std::vector<double> udfT_host[2][3];
    double *tface = nullptr;           // thermal wall pass: one value per face-node entry
    long long n_tface = 0;
    void *ttmp = nullptr;              // thermal level-set pass: node-sized scratch (R)
    // sort
    SortBufs sb;
    long long *staging = nullptr;      // P2G partial node blocks (fixed point)
    double *stage = nullptr;           // one FP64 particle field: host transfers
    long long stage_cap = 0;
    size_t staging_cap = 0;            // in tiles
    int nch = 7;
    // control block
    Ctl *ctl = nullptr;                // device
    Ctl *ctl_host = nullptr;           // pinned mirror
    unsigned long long *bounds_cur = nullptr;  // device: bounds used by this step's P2G
    unsigned long long *bounds2 = nullptr;     // device: bounds of the MUSL re-projection
    unsigned long long *dtmin2 = nullptr;      // device: scratch min
    double *diag_dev = nullptr;
    // state
    bool parts_sorted = false;         // perm valid for the current storage order
    bool reduce_stale = true;          // ctl reductions need recomputing
    double host_time = 0.0, host_dt = 0.0;
    long long host_steps = 0;
    // CUDA graph of one fused step
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // one per buffer orientation
    bool warm[2] = {false, false};
    int orient = 0;                                 // 1 when pa holds the second allocation
    cudaEvent_t ev[6] = {};
    double stage_ms[5] = {};
    bool timing = false;
    // launch variants of the P2G and fused G2P kernels (rows per pass and
    // threads per block; every variant gives bit-identical results), chosen
    // by the autotuner (exg_autotune) or set by exg_set_variants
    int p2g_var = 0, g2p_var = 0;
    bool tuned = false;
    // the particles are in the order a fused step leaves them (tile-major,
    // as every later step sees them): set by exg_step, cleared by uploads
    bool reordered = false;
    // TMA staging of the fused G2P's node blocks: the tensor map over the
    // nodal records (Nodes::rec), when the grid has no periodic axis
    bool tma = false;
    CUtensorMap tmap;
    void *rec = nullptr;
    double tune_ms[2][4] = {};   // measured ms of each variant: [p2g/g2p][variant]

    template <class R>
    Parts<R> &A() { return *reinterpret_cast<Parts<R> *>(pa); }
    template <class R>
    Parts<R> &Bp() { return *reinterpret_cast<Parts<R> *>(pb); }
    template <class R>
    Nodes<R> &N() { return *reinterpret_cast<Nodes<R> *>(nodes); }
};

#define EXG_CUDA_OK(call)                                                              \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " +    \
                                                        cudaGetErrorString(e_));       \
    } while (0)

}  // namespace exg

// Internal plan layout shared by the operator and solver translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <functional>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/iga_mf.h"
#include "iga_device.cuh"
#include "iga_host.hpp"

namespace iga {

// Device data of one operator precision.
struct OperatorData {
    bool ready = false;
    int warps = 8;
    StripGrid grid;         // strips of this operator (a MIXED plan's two operators may differ in TY)
    void *tabX = nullptr;   // [NSX][2][NQ][NB][32]
    void *tabY = nullptr;   // [ney][2][NQ][NB]
    void *G = nullptr;      // precomputed geometry (may be null)
    void *frame = nullptr;  // seam frames
    void *wq = nullptr;     // [NQ*NQ] quadrature weight products
    void *kappa = nullptr;  // on-the-fly coefficient
    void *CP = nullptr;     // on-the-fly control points in the operator precision
    size_t geom_bytes = 0;
};

struct SolverState;   // defined by the solver translation unit

// One plan's precomputed-geometry set-up inside a batch's single launch:
// G in FP64 and / or FP32 (null: not wanted) on strip grid g from the plan's
// FP64 tables and control points; t0 = the job's first point in the launch.
struct GeomJob {
    double *G64 = nullptr;
    float *G32 = nullptr;
    const double *tx = nullptr, *ty = nullptr, *cp = nullptr, *qw = nullptr, *kappa = nullptr;
    StripGrid g;
    int *err = nullptr;
    long long t0 = 0;
};

// Device memory of many plans carved out of a few large allocations. A batch
// creates hundreds of small plans; with one cudaMalloc per table and a device
// synchronisation per plan their set-up cost far more than the solves.
// While plan_arena() is set on a thread, plan creation allocates from that
// arena and skips its synchronisations (the caller synchronises once and
// checks every plan's error flag); the plans' destroy leaves arena memory
// alone, and the arena's owner releases it after destroying the plans.
struct PlanArena {
    std::vector<std::pair<char *, size_t>> chunks;
    size_t used = 0;   // bytes used in the last chunk
    cudaError_t alloc(void **p, size_t bytes);
    bool owns(const void *p) const;
    void release();
    // Deferred mode (defer = true): buffers with host data come from a data
    // region of chunks with host shadows; upload() copies into the shadow.
    // A chunk that is full and completely written is sent to the device by a
    // copy thread while the plans are still being built (a copy from pageable
    // memory runs at about 11 GB/s however many threads issue it, so it is
    // overlapped with the plans' host work rather than split); flush() sends
    // the rest, then runs the plans' geometry set-up (one launch over all of
    // them). Building many plans then makes no synchronising copy per buffer.
    bool defer = false;
    mutable std::mutex mu;   // plans may be built by several host threads at once
    struct DataChunk {
        char *dev = nullptr;
        std::unique_ptr<char[]> host;   // the shadow
        size_t size = 0, used = 0, staged = 0;   // bytes allocated / written into the shadow
        bool sealed = false;            // no further allocations
        bool taken = false;             // copied (or being copied)
    };
    std::vector<std::unique_ptr<DataChunk>> dchunks;
    std::vector<std::pair<char *, size_t>> dblocks;   // the device memory the chunks are carved from
    size_t dblock_used = 0;
    std::condition_variable cv;
    std::thread copier;
    bool copier_stop = false;
    cudaError_t copy_err = cudaSuccess;
    // Copies from host memory that outlives the flush (a plan's own control
    // points) into buffers of the plain region, done by the copy thread
    // without staging: defer_copy() queues one.
    struct DirectCopy {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<DirectCopy> direct;
    const void *copying = nullptr;   // source of the direct copy in progress
    void defer_copy(void *dst, const void *src, size_t bytes);
    // Forgets the queued copies from [lo, hi) and waits for one in progress
    // (a plan destroyed before the flush).
    void drop_copies(const void *lo, const void *hi);
    void seal_last(bool start_copier);   // with mu held
    void copy_loop(int device);
    void stop_copier();
    ~PlanArena() { stop_copier(); }
    // deferred geometry set-up: one job per plan (a MIXED plan's two
    // precisions on the same strips share one), all run by one launch in flush()
    std::vector<GeomJob> geom;
    cudaError_t alloc_data(void **p, size_t bytes);
    void stage(void *dst, const void *src, size_t bytes);
    void defer_geom(const GeomJob &j);
    cudaError_t flush();
};
PlanArena *&plan_arena();

void set_error(const std::string &s);
const std::string &last_error();

// Checks of a reference-shaped call's d_IEN / d_ID (refentry_check_kernel):
// flag bits, the stream-ordered launcher (flags: one device int; seen:
// (m n + 31) / 32 device words; nothing is allocated) and the status the
// flags mean (IGA_OK when the call can run, kCheckIDOrder alone included).
enum { kCheckIEN = 1, kCheckIDOrder = 2, kCheckIDRange = 4, kCheckIDTwice = 8 };
int refentry_check(const int *IEN, const int *ID, int p, int nex, int ney, unsigned *seen, int *flags,
                   cudaStream_t s);
int refentry_status(int flags);

// Largest warps per CTA of the apply kernel for degree P, precision
// (IGA_FP64 / IGA_FP32) and geometry mode that fits the shared-memory budget.
int warps_for(int P, int prec, int geom);

}  // namespace iga

struct iga_plan {
    int p = 0, nex = 0, ney = 0, m = 0, n = 0;
    long long nfunc = 0;
    int precision = IGA_FP64, geometry = IGA_GEOM_PRECOMPUTED, sign = IGA_SIGN_REFERENCE, bc = IGA_BC_REFERENCE;
    int device = 0;
    iga::StripGrid grid{};
    iga::Patch patch;
    iga::OperatorData op64, op32;
    double *tabX64 = nullptr, *tabY64 = nullptr, *CP = nullptr, *qw = nullptr;
    int *d_err = nullptr;
    double *kappa_dev = nullptr;   // coefficient at the quadrature points (null: 1)
    int kappa_version = 0;         // bumped by every change of kappa
    double *h_stage_x = nullptr, *d_stage_x = nullptr, *d_stage_y = nullptr;
    // iga_apply_host's pipeline: copy-in, compute and copy-out streams, one
    // event per slab and stage, and the start event
    cudaStream_t host_st[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t host_ev[2][16] = {};
    cudaEvent_t host_ev0 = nullptr;
    void *h_pinned = nullptr;
    iga::SolverState *solver = nullptr;
    // Equation number of every control point (the reference's ID array) when
    // the reference-shaped entry point was given one other than the natural
    // order with -1 on the boundary ring; null otherwise.
    int *eq_id = nullptr;
    // Polls of the apply kernel's bounded waits (< 0: the default limit).
    long long wait_polls = -1;
    // The exact FEM preconditioner may split its x transforms by parity.
    bool pc_split = true;
    // The solver runs its iterations inside a conditional-loop graph.
    bool solver_graph = true;
    // Arena the plan's creation-time buffers came from (not owned), or null.
    iga::PlanArena *arena = nullptr;
};

int iga_apply_internal(iga_plan *pl, int prec, const void *x, void *y, cudaStream_t s);
// Operator with explicit sign / boundary rule (the solver applies +K with identity rows).
int iga_apply_internal_sb(iga_plan *pl, int prec, const void *x, void *y, cudaStream_t s, int sign, int bc);
int iga_check_error_flag(iga_plan *pl);
// Computes G of one operator precision from the plan's tables and kappa (device).
int iga_rebuild_geometry(iga_plan *pl, cudaStream_t s);
void iga_solver_release(iga_plan *pl);

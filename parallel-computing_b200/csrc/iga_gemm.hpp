// Dense GEMMs of the exact FEM preconditioner (the two transforms by the
// x-direction eigenvectors), written for sm_100a without a BLAS library:
//   - FP32 data on the 5th-generation tensor cores (tcgen05.mma kind::tf32,
//     accumulator in TMEM), operand tiles brought into shared memory by the
//     tensor-memory accelerator (cp.async.bulk.tensor, 128-byte swizzle);
//   - FP64 data on the FP64 tensor cores (DMMA, mma.sync f64).
// C[m][n] = sum_k A(m, k) B(n, k), C row-major with leading dimension ldc;
// each operand is either K-major (X[row][k], k contiguous) or MN-major
// (X[k][row], row contiguous), with a leading dimension in elements.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace iga {

// A block-diagonal operand split at kb (> 0, a multiple of 16): the operand
// indexed by the split dimension (M with on_n false, N with on_n true) has
// nonzeros only in the blocks [0, kb) x [0, kb) and [kb, K) x [kb, K) of
// (that index, k). The tiles along that dimension are laid out block by
// block, each running its k loop over its own block's range only.
struct GemmSplit {
    int kb = 0;
    bool on_n = false;
};

struct GemmOperand {
    const void *ptr = nullptr;
    int ld = 0;           // elements between consecutive outer-index entries
    bool mn_major = false;
};

// A prepared FP32 (TF32 tensor core) GEMM: tensor maps built once for fixed
// operand addresses and sizes; launching it is graph-capturable.
struct GemmTF32 {
    CUtensorMap ta, tb;
    bool a_mn = false, b_mn = false;
    int M = 0, N = 0, K = 0;       // logical sizes (tiles, k slices)
    int Mst = 0, Nst = 0;          // rows / columns of C written (>= M, N: padding written as zeros)
    float *C = nullptr;
    int ldc = 0;
    int bn = 128;                  // output tile width (128, or 64 for small products)
    GemmSplit split;               // block-diagonal operand, if any
    // 1 (A) or 2 (B): an operand that no kernel launched on the same stream
    // writes (the eigenvectors), whose first tiles a launch with a programmatic
    // dependency may fetch before the preceding grid has finished; 0: none
    int const_op = 0;
    bool ready = false;
};

// Builds the tensor maps (returns IGA_OK or an IGA_ERR_* status with the
// message recorded). The operand extents are the K-major / MN-major storage
// extents: rows = M (or N) and K for the logical problem; reads past them
// are zero-filled by the copy engine.
int gemm_tf32_prepare(GemmTF32 &g, GemmOperand A, GemmOperand B, float *C, int ldc, int M, int N, int K, int Mst,
                      int Nst, GemmSplit split = GemmSplit());
// Where a GEMM's result goes instead of C: element (r, c) with r < rows,
// c < cols is stored at out[(r + 1) ld + c + 1] (the interior block of a
// vector on an (rows + 2) x ld grid of control points), in FP32 or FP64,
// multiplied by sqrt(*rr) when rr is set and *rr is positive and finite.
struct GemmScatter {
    void *out = nullptr;
    bool f64 = false;
    int ld = 0, rows = 0, cols = 0;
    const double *rr = nullptr;
};

// Stream-ordered launch; a bounded wait that gives up sets *err to
// IGA_ERR_TIMEOUT (the kernel then drains its copies and MMAs and returns).
// With sc.out set the result is scattered as GemmScatter says and C is not written.
int gemm_tf32_launch(const GemmTF32 &g, cudaStream_t s, int *err, const GemmScatter &sc = GemmScatter());

// FP64 GEMM on DMMA tiles, same operand conventions (no tensor maps: the
// tiles are staged by cp.async). Mst/Nst as above; with sc.out set (FP64
// output only) the result is scattered instead of written to C.
int gemm_f64_launch(GemmOperand A, GemmOperand B, double *C, int ldc, int M, int N, int K, int Mst, int Nst,
                    cudaStream_t s, const GemmScatter &sc = GemmScatter(), GemmSplit split = GemmSplit());
// CTA shape of the FP64 GEMM for every later launch (0: 128 x 128, 1: 128 x 64,
// 2: 64 x 64; -1: the default, 2). For timing the shapes.
void gemm_f64_force_shape(int shape);

}  // namespace iga

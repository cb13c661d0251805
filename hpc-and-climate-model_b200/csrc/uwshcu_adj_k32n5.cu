// uwshcu_adj_k32n5.cu -- the adjoint kernels for mkx + 1 <= 32 levels and ncnst <= 5 tracers, with
// this unit's constant bank and launch hooks.  Built without FMA contraction (values = FP64 path).
#include "uwshcu_adj_kernel.cuh"

extern "C" cudaError_t uw_adj_set_constants_k32n5(const UwConst* h, const double* tbl)
{
    cudaError_t e = cudaMemcpyToSymbol(c, h, sizeof(UwConst));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_estbl, tbl, sizeof(double) * UW_TBL);
}

static UwAdj to_dev(const UwAdjHost& h)
{
    UwAdj g;
    g.wl = h.wl;
    g.b0 = h.b0;
    g.nb = h.nb;
    g.ab = static_cast<int2*>(h.ab);
    g.d = static_cast<double2*>(h.d);
    g.rcap = h.rcap;
    g.ids = h.ids;
    g.cap = h.cap;
    g.nrow = h.nrow;
    g.ovf = h.ovf;
    g.adj = h.adj;
    g.astride = h.astride;
    g.status = h.status;
    g.split = h.split;
    g.gsave = h.gsave;
    g.defect = h.defect;
    return g;
}

// phase 0: forward sweep of slots [0, nb) in blocks of UW_ADJ_BLOCK threads; phase 1: reverse sweep,
// one warp per tape, in blocks of UW_ADJ_RBLOCK threads.
extern "C" cudaError_t uw_adj_launch_k32n5(const UwArgs* a, const void* slots, const uwshcu_adjoint* c,
                                           int phase, cudaStream_t stream)
{
    const UwAdjHost& h = *static_cast<const UwAdjHost*>(slots);
    if (h.nb <= 0) return cudaSuccess;
    const UwAdj g = to_dev(h);
    if (phase == 0) {
        const dim3 grid((unsigned)((h.nb + UW_ADJ_BLOCK - 1) / UW_ADJ_BLOCK));
        uwshcu_adj_forward<32, 5><<<grid, UW_ADJ_BLOCK, 0, stream>>>(*a, g);
    } else {
        const dim3 grid((unsigned)((h.nb + UW_ADJ_RBLOCK - 1) / UW_ADJ_RBLOCK));
        uwshcu_adj_reverse<32, 5><<<grid, UW_ADJ_RBLOCK, 0, stream>>>(*a, g, *c);
    }
    return cudaGetLastError();
}

// bytes of one tape row of a warp: 32 records of operand indices and partials
extern "C" size_t uw_adj_row_bytes_k32n5() { return 32 * (sizeof(int2) + sizeof(double2)); }

// Warps of the forward sweep (one per block) that one SM holds at once.
extern "C" cudaError_t uw_adj_forward_occupancy_k32n5(int* warps_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(warps_per_sm, uwshcu_adj_forward<32, 5>, UW_ADJ_BLOCK, 0);
}

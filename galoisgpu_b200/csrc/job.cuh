// job.cuh -- device side of one batched or served query (BatchJob): its
// traversal parameters inside a scratch arena and its result record.
// Shared by the batched kernel (batch.cu) and the resident serving kernel
// (resident.cu).
#pragma once
#include "frontier.cuh"
#include "gft_internal.h"

namespace gft {
namespace dev {

// Parameters of one job's traversal inside the batch scratch.
__device__ __forceinline__ TravParams job_params(const BatchJob &jb, char *scratch, uint32_t hub_degree,
                                                 TraversalCtl *ctl)
{
    char *base = scratch + jb.scratch;
    const size_t qbytes = ((size_t)jb.nnodes * 4 + 255) & ~(size_t)255;
    TravParams p{};
    p.row_start = jb.row_start;
    p.edge_dst = jb.edge_dst;
    p.edge_data = jb.edge_data;
    p.nnodes = jb.nnodes;
    p.src = jb.src;
    p.out = jb.out;
    p.q[0] = reinterpret_cast<uint32_t *>(base);
    p.q[1] = reinterpret_cast<uint32_t *>(base + qbytes);
    p.hub_cap = jb.hub_cap;
    p.hub_degree = hub_degree;
    p.qcap = jb.nnodes;
    p.delta = jb.delta;
    p.ctl = ctl;
    p.skip_block = -1;
    p.vec_ok = jb.vec_ok;
    p.uniform = jb.uniform;
    p.nedges = jb.nedges;
    p.dir_opt = jb.dir_opt;
    if (jb.app == 1) {
        p.far[0] = reinterpret_cast<uint32_t *>(base + 2 * qbytes);
        p.far[1] = reinterpret_cast<uint32_t *>(base + 3 * qbytes);
        p.qstamp = reinterpret_cast<uint32_t *>(base + 4 * qbytes);
        p.hubs = reinterpret_cast<uint2 *>(base + 5 * qbytes);
    } else {
        const size_t vbytes = ((size_t)((jb.nnodes + 31) / 32) * 4 + 255) & ~(size_t)255;
        p.parent = jb.parent;
        p.visited = reinterpret_cast<uint32_t *>(base + 2 * qbytes);
        p.hubs = reinterpret_cast<uint2 *>(base + 2 * qbytes + vbytes);
    }
    return p;
}

__device__ __forceinline__ void write_result(BatchJob &r, const TraversalCtl &c, unsigned long long t0)
{
    r.status = c.error;
    r.error_where = c.error_where;
    r.levels = c.levels;
    r.iterations = c.iterations;
    r.edges = c.edges;
    r.t_start = t0;
    r.t_end = globaltimer_ns();
}

}  // namespace dev
}  // namespace gft

// mp_graph.cuh -- building CUDA graphs with device-controlled while loops.
//
// A graph is a chain of segments.  A captured segment is a stream capture of
// ordinary kernel launches recorded directly into the graph.  A while segment is
// a conditional node whose body is built by a nested builder; kernels in the
// graph set the loop condition with cudaGraphSetConditional, so a Krylov
// solve runs to convergence inside one graph launch with no host round trip.
#pragma once
#include <functional>
#include <vector>
#include "mp_common.cuh"

namespace mp {

long long launch_counter();

struct GraphBuilder {
    cudaGraph_t g = nullptr;
    cudaGraphNode_t last = nullptr;
    cudaStream_t s = nullptr;  // capture stream (a private non-blocking stream)
    int depth = 0;             // while-loop nesting level of this builder
    int *counts = nullptr;     // kernels captured per nesting level (optional, >= 3 ints)

    int init_root(cudaStream_t cap) {
        s = cap;
        MP_CUDA(cudaGraphCreate(&g, 0));
        return MP_OK;
    }

    // append the kernels launched by `fn` (fn issues them on `s`), captured
    // straight into this graph after `last` so that kernels setting a loop
    // condition live in the same graph as the conditional node
    int captured(const std::function<int(cudaStream_t)> &fn) {
        MP_CUDA(cudaStreamBeginCaptureToGraph(s, g, last ? &last : nullptr, nullptr, last ? 1 : 0,
                                              cudaStreamCaptureModeThreadLocal));
        const long long c0 = launch_counter();
        int rc = fn(s);
        if (counts && depth < 3)
            counts[depth] += (int)(launch_counter() - c0);
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps);
        std::vector<cudaGraphNode_t> leaves;
        if (e == cudaSuccess && deps)
            leaves.assign(deps, deps + ndeps);
        cudaGraph_t out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(s, &out);
        if (rc != MP_OK)
            return rc;
        if (e != cudaSuccess || e2 != cudaSuccess)
            return fail(MP_CUDA_ERROR, "stream capture failed: %s",
                        cudaGetErrorString(e != cudaSuccess ? e : e2));
        if (leaves.size() == 1) {
            last = leaves[0];
        } else if (!leaves.empty()) {  // join several leaves
            cudaGraphNode_t j;
            MP_CUDA(cudaGraphAddEmptyNode(&j, g, leaves.data(), leaves.size()));
            last = j;
        }
        return MP_OK;
    }

    // a handle for a while loop; default value 0 is re-applied at each launch
    int make_handle(cudaGraphConditionalHandle *h) {
        MP_CUDA(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
        return MP_OK;
    }

    // append `while (cond) body`; the body is populated through a nested builder
    int while_loop(cudaGraphConditionalHandle h, const std::function<int(GraphBuilder &)> &body) {
        cudaGraphNodeParams p = {};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        MP_CUDA(cudaGraphAddNode(&node, g, last ? &last : nullptr, last ? 1 : 0, &p));
        GraphBuilder b;
        b.g = p.conditional.phGraph_out[0];
        b.s = s;
        b.depth = depth + 1;
        b.counts = counts;
        MP_TRY(body(b));
        last = node;
        return MP_OK;
    }
};

// Executable graph owned by a handle
struct GraphExec {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~GraphExec() { reset(); }
    void reset() {
        if (e)
            cudaGraphExecDestroy(e);
        if (g)
            cudaGraphDestroy(g);
        e = nullptr;
        g = nullptr;
    }
    int instantiate(GraphBuilder &b) {
        reset();
        g = b.g;
        b.g = nullptr;
        MP_CUDA(cudaGraphInstantiate(&e, g, 0));
        return MP_OK;
    }
    int launch(cudaStream_t s) {
        MP_CUDA(cudaGraphLaunch(e, s));
        count_launch();
        return MP_OK;
    }
};

}  // namespace mp

// mp_graph.cuh -- building CUDA graphs with device-controlled while loops.
//
// A graph is a chain of segments.  A captured segment is a stream capture of
// ordinary kernel launches, added as a child-graph node.  A while segment is
// a conditional node whose body is built by a nested builder; kernels in the
// graph set the loop condition with cudaGraphSetConditional, so a Krylov
// solve runs to convergence inside one graph launch with no host round trip.
#pragma once
#include <functional>
#include "mp_common.cuh"

namespace mp {

struct GraphBuilder {
    cudaGraph_t g = nullptr;
    cudaGraphNode_t last = nullptr;
    cudaStream_t s = nullptr;  // capture stream (a private non-blocking stream)

    int init_root(cudaStream_t cap) {
        s = cap;
        MP_CUDA(cudaGraphCreate(&g, 0));
        return MP_OK;
    }

    // append the kernels launched by `fn` (fn issues them on `s`)
    int captured(const std::function<int(cudaStream_t)> &fn) {
        cudaGraph_t tmp = nullptr;
        MP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int rc = fn(s);
        cudaError_t e = cudaStreamEndCapture(s, &tmp);
        if (rc != MP_OK) {
            if (tmp)
                cudaGraphDestroy(tmp);
            return rc;
        }
        if (e != cudaSuccess)
            return fail(MP_CUDA_ERROR, "stream capture failed: %s", cudaGetErrorString(e));
        cudaGraphNode_t node;
        e = cudaGraphAddChildGraphNode(&node, g, last ? &last : nullptr, last ? 1 : 0, tmp);
        cudaGraphDestroy(tmp);
        if (e != cudaSuccess)
            return fail(MP_CUDA_ERROR, "cudaGraphAddChildGraphNode: %s", cudaGetErrorString(e));
        last = node;
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

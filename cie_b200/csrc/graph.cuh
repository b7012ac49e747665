// Device-driven solver loops: a CUDA graph whose single node is a WHILE
// conditional node (CUDA 12.4+).  The body is captured from the launches that
// `body(handle)` issues on the given stream; kernels of the body end the loop
// with cudaGraphSetConditional(handle, 0).  The condition resets to 1 at every
// launch of the graph, so each launch runs the body until a kernel clears it.
#pragma once

#include "common.cuh"

#include <cstdlib>

namespace ciecu {

// CIECU_GRAPH_LOOP=0 selects the plain captured-chunk graphs (same kernels,
// host-polled) -- profilers cannot attribute kernels inside conditional graphs.
inline bool device_loop_enabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("CIECU_GRAPH_LOOP");
        return !(v && v[0] == '0');
    }();
    return enabled;
}

template <typename F>
int build_while_graph(cudaStream_t st, F&& body, cudaGraphExec_t* exec) {
    *exec = nullptr;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle handle = 0;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams params{};
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) {
        params.type = cudaGraphNodeTypeConditional;
        params.conditional.handle = handle;
        params.conditional.type = cudaGraphCondTypeWhile;
        params.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &params);
    }
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "while-loop graph node");
    }
    cudaGraph_t bodyGraph = params.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(st, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "while-loop body capture");
    }
    const int status = body(g, handle);
    e = cudaStreamEndCapture(st, &bodyGraph);
    if (status != CIECU_OK || e != cudaSuccess) {
        cudaGraphDestroy(g);
        return status != CIECU_OK ? status : cuda_fail(e, "while-loop body capture end");
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "while-loop graph instantiate");
    return CIECU_OK;
}

// Inside a capture on `st`: appends IF(handle) { body on st2 } after the work
// captured so far; later work on `st` depends on the conditional node.
template <typename F>
int capture_if(cudaStream_t st, cudaStream_t st2, cudaGraphConditionalHandle handle, F&& body) {
    cudaStreamCaptureStatus cs;
    unsigned long long id = 0;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CIECU_CUDA(cudaStreamGetCaptureInfo(st, &cs, &id, &cg, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(CIECU_ERR_CUDA, "capture_if: stream is not capturing");
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeIf;
    params.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    CIECU_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &params));
    CIECU_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t ib = params.conditional.phGraph_out[0];
    CIECU_CUDA(cudaStreamBeginCaptureToGraph(st2, ib, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int status = body(st2);
    cudaError_t e = cudaStreamEndCapture(st2, &ib);
    if (status != CIECU_OK) return status;
    if (e != cudaSuccess) return cuda_fail(e, "capture_if: body capture end");
    return CIECU_OK;
}

}  // namespace ciecu

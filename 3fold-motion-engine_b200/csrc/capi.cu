// Library-wide C entry points: version and the per-thread error message.
#include "b2c_barrier.cuh"
#include "b2c_common.cuh"

namespace b2c {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

}  // namespace b2c

extern "C" int32_t b2c_version(void) { return 100; }
extern "C" int32_t b2c_barrier_words(void)
{
    static_assert(b2c::kBarrierWords == B2C_BARRIER_WORDS, "the header's barrier size");
    return b2c::kBarrierWords;
}
extern "C" const char *b2c_last_error(void) { return b2c::g_err; }

static int count_kernel_nodes(cudaGraph_t g, int depth)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return -1;
    if (n == 0) return 0;
    cudaGraphNode_t *nodes = new cudaGraphNode_t[n];
    int total = 0;
    if (cudaGraphGetNodes(g, nodes, &n) != cudaSuccess) total = -1;
    for (size_t i = 0; i < n && total >= 0; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) != cudaSuccess) {
            total = -1;
            break;
        }
        if (t == cudaGraphNodeTypeKernel) {
            ++total;
        } else if (t == cudaGraphNodeTypeGraph && depth < 8) {
            cudaGraph_t child;
            if (cudaGraphChildGraphNodeGetGraph(nodes[i], &child) != cudaSuccess) {
                total = -1;
                break;
            }
            const int c = count_kernel_nodes(child, depth + 1);
            total = c < 0 ? -1 : total + c;
        }
    }
    delete[] nodes;
    return total;
}

extern "C" int32_t b2c_graph_kernel_nodes(void *graph)
{
    if (!graph) {
        b2c::set_error("b2c_graph_kernel_nodes: null graph");
        return -1;
    }
    const int n = count_kernel_nodes(reinterpret_cast<cudaGraph_t>(graph), 0);
    if (n < 0) b2c::set_error("b2c_graph_kernel_nodes: %s", cudaGetErrorString(cudaGetLastError()));
    return n;
}

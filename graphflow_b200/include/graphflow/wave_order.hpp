// Node order of a device-resident wave (device_flow.cuh). A transform forwards all its chunks to
// one node, so when that node runs later in the same wave the chunks join its input of this wave
// instead of the next one's. The order puts the successor after the transform along every such
// edge that no cycle of transforms alone forbids: a run of transforms and the node after them then
// take one wave. Nodes on a cycle of transforms alone keep their index order. Host code only.
#pragma once

#include <cstdint>
#include <vector>

namespace graphflow {
namespace devflow {

// forwards[k] != 0: node k forwards every input chunk to succ[k] (succ[k] >= N or == k: no such
// edge). Returns a permutation of 0 .. N-1: the order in which a wave runs the nodes.
inline std::vector<std::uint32_t> waveOrder(const std::vector<char>& forwards, const std::vector<std::uint32_t>& succ)
{
    const auto N = static_cast<std::uint32_t>(forwards.size());
    auto edge = [&](std::uint32_t k) { return forwards[k] != 0 && k < succ.size() && succ[k] < N && succ[k] != k; };
    std::vector<std::uint32_t> indeg(N, 0u), seq;
    seq.reserve(N);
    for (std::uint32_t k = 0; k < N; ++k)
        if (edge(k))
            ++indeg[succ[k]];
    std::vector<char> placed(N, 0);
    // walk each chain of transform edges from a node no transform feeds: the walk continues into
    // a successor once its last transform predecessor is placed
    for (std::uint32_t k = 0; k < N; ++k)
        for (std::uint32_t v = k; indeg[v] == 0u && !placed[v];) {
            placed[v] = 1;
            seq.push_back(v);
            if (!edge(v))
                break;
            v = succ[v];
            if (indeg[v] != 0u)
                --indeg[v];
        }
    for (std::uint32_t k = 0; k < N; ++k)
        if (!placed[k])
            seq.push_back(k);
    return seq;
}

} // namespace devflow
} // namespace graphflow

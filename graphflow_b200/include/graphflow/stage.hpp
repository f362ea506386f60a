// The hook protocol of an execution stage (the reference's StageBase, flow/Execution.hpp:1538-1561):
// launch -> [advance]* -> finish | abort, and the batch a stage receives. Host-only, so the
// scheduler and its tests compile without the device code.
#pragma once

#include <cstddef>
#include <cstdint>
#include <deque>
#include <vector>

#include <cuda_runtime_api.h>

#include "core.hpp"

namespace graphflow {

struct Batch {
    std::vector<ChunkDescriptor> chunks;
    std::uint64_t firstId = 0u;
    std::uint64_t particles() const
    {
        std::uint64_t n = 0;
        for (const auto& c : chunks)
            n += c.fill;
        return n;
    }
};

class Stage {
public:
    virtual ~Stage() = default;
    // Enqueue the batch's first device stage on `s`. Returns the output chunks it acquired.
    virtual std::uint32_t launch(cudaStream_t s, const Batch& b) = 0;
    // Called after the last enqueued device work completed. Returns true when it enqueued more;
    // `allocated` receives the output chunks acquired by this call.
    virtual bool advance(cudaStream_t s, const Batch& b, std::uint32_t& allocated) = 0;
    // Publish the batch's outputs (Execution.hpp:2457-2461).
    virtual void finish(const Batch& b, std::vector<ChunkDescriptor>& outputs) = 0;
    // Release every unpublished output; the stage is single-use afterwards (Execution.hpp:2652-2656).
    virtual void abort() = 0;
    virtual std::uint64_t launches() const { return m_launches; }
    // A stage that sizes its own batches (a partition group) answers true and plans them:
    // planBatch returns how many chunks of `ready` (a prefix) to take with at most `available`
    // output chunks reserved, and the reservation in `reserve`; 0 takes nothing. Other stages
    // leave batch sizing to the runner.
    virtual bool plansBatches() const { return false; }
    virtual std::size_t planBatch(const std::deque<ChunkDescriptor>&, std::uint32_t, std::uint32_t& reserve) const
    {
        reserve = 0u;
        return 0u;
    }
    // Partition batches the last launch ran (a partition group runs several per launch).
    virtual std::uint32_t lastLaunchBatches() const { return 1u; }
    // A stage whose device work reports its own completion in host memory answers true; the
    // runner then polls completed() instead of recording and querying the node's event.
    virtual bool pollsCompletion() const { return false; }
    virtual bool completed() const { return true; }

protected:
    std::uint64_t m_launches = 0;
};

} // namespace graphflow

// graphflow_b200_particle_feedback: a command-line drop-in for the reference example binary
// graphFlow_particle_feedback (examples/particle_feedback/main.cpp and Cli.hpp). It takes the same
// flags and prints the same report: "# ..." provenance lines, "# weight,count", the sorted
// histogram rows "weight,count" and "# non-terminating K" when the visit cap stopped K particles
// (main.cpp:22-33, 48-58). The run goes through this library's C ABI: the feedback graph through
// the Flow (gf_run_particle_feedback) on the current CUDA device, then the sorted histogram on the
// device (gf_histogram_u32) instead of the reference's host sort.
//
// C, P and T the command line leaves out come from the device policy (gf_device_policy, the
// reference's makeDevicePolicy rules) with the accelerator ratio P/C = 8 unless an explicit C is
// below the logical tile width, as Cli.hpp resolveOptions does; an explicit P above the run size or
// the payload budget is a command-line error there and here.
//
// Differences, by design: only --backend cuda runs (there is no CPU or other backend); T shapes
// the policy's C (a multiple of T) but the partition kernels keep their own 1024-particle tiles.
// Flags that configure parts of the reference this build does not have (frame cap, occupancy
// target, pool budget and mode, per-chunk transform schedule) are parsed and checked as the
// reference does and reported as inert on stderr. The kernel workload (--workload kernel,
// KernelAxes.hpp runKernelAxes) runs through gf_run_kernel_axes with 64, 1024, 4096 or 65536 ports
// on the dense or the hash bin path.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "cli_common.hpp"
#include "graphflow_b200.h"

namespace {

using gfcli::cudaOrThrow;
using gfcli::expectOneOf;
using gfcli::lastError;
using gfcli::parseU32;
using gfcli::parseU64;

constexpr const char* kName = "graphflow_b200_particle_feedback";
constexpr std::uint32_t kAcceleratorLivePerChunk = 8u; // DevicePolicy.hpp:53
constexpr std::uint32_t kLogicalTileWidth = 128u;      // DevicePolicyConfig::logicalTileWidth

struct Options {
    bool help = false;
    std::string backend = "cpu"; // the reference's default; this build runs only "cuda"
    std::uint64_t particles = 0u;
    std::optional<std::uint32_t> chunkSize, liveParticles, tileSize;
    std::uint32_t batchChunks = 1u;
    std::uint64_t seed = 0u;
    std::uint32_t maxVisits = 64u;
    std::uint32_t device = 0u;
    std::string workload = "feedback";
    std::vector<std::string> inert;     // accepted for CLI parity, no effect here
    std::vector<std::string> kernelOnly; // flags of the kernel workload
    std::string scatter = "shared", binPath = "dense", distribution = "balanced"; // KernelOptions defaults
    std::uint32_t bins = 64u;
    bool deviceResident = false; // B200 extension: the Flow run device-resident
};

void usage(std::ostream& out)
{
    out << "usage: " << kName << " --backend cuda [--device D]\n"
           "                                        [--particles N] [--chunk-size C]\n"
           "                                        [--live-particles P] [--tile-size T]\n"
           "                                        [--batch-chunks Q] [--seed S] [--max-visits M]\n"
           "                                        [--workload feedback|kernel] [--device-resident]\n"
           "       kernel workload only: [--scatter shared|direct] [--bin-path dense|hash]\n"
           "                             [--bins 64|1024|4096|65536]\n"
           "                             [--distribution balanced|one-hot|skewed|sparse]\n"
           "       accepted for parity with graphFlow_particle_feedback, no effect here:\n"
           "       [--frame-cap F] [--occupancy-target D] [--pool-budget-bytes B]\n"
           "       [--pool-mode fixed|slotArena] [--slot-arena-budget BYTES]\n"
           "       [--chunk-kernel-schedule off|perChunk] [--chunk-queue-depth D]\n"
           "       [--chunk-latency-cap-us U]\n"
           "       defaults: C, P and T from the device policy (the reference's rules), Q = 1,\n"
           "       seed 0, 64 visits.\n"
           "       Output: '# ...' lines, '# weight,count', then one 'weight,count' row per distinct\n"
           "       final weight in ascending order, and '# non-terminating K' if K particles hit the cap.\n";
}

Options parse(int argc, char** argv)
{
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string flag = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc)
                throw std::invalid_argument(flag + ": missing value");
            return argv[++i];
        };
        if (flag == "--help" || flag == "-h") {
            o.help = true;
            return o;
        } else if (flag == "--backend") {
            o.backend = next();
        } else if (flag == "--particles") {
            o.particles = parseU64(flag, next());
        } else if (flag == "--chunk-size") {
            o.chunkSize = parseU32(flag, next());
        } else if (flag == "--live-particles") {
            o.liveParticles = parseU32(flag, next());
        } else if (flag == "--tile-size") {
            o.tileSize = parseU32(flag, next());
        } else if (flag == "--batch-chunks") {
            o.batchChunks = parseU32(flag, next());
        } else if (flag == "--seed") {
            o.seed = parseU64(flag, next());
        } else if (flag == "--max-visits") {
            o.maxVisits = parseU32(flag, next());
        } else if (flag == "--device") {
            o.device = parseU32(flag, next(), true);
        } else if (flag == "--device-resident") {
            o.deviceResident = true;
        } else if (flag == "--workload") {
            o.workload = next();
            expectOneOf(flag, o.workload, {"feedback", "kernel"});
        } else if (flag == "--frame-cap" || flag == "--occupancy-target" || flag == "--chunk-queue-depth") {
            parseU32(flag, next());
            o.inert.push_back(flag);
        } else if (flag == "--chunk-latency-cap-us") {
            parseU32(flag, next(), true);
            o.inert.push_back(flag);
        } else if (flag == "--pool-budget-bytes" || flag == "--slot-arena-budget") {
            if (parseU64(flag, next()) == 0u)
                throw std::invalid_argument(flag + ": value must be non-zero");
            o.inert.push_back(flag);
        } else if (flag == "--pool-mode") {
            expectOneOf(flag, next(), {"fixed", "slotArena"});
            o.inert.push_back(flag);
        } else if (flag == "--chunk-kernel-schedule") {
            expectOneOf(flag, next(), {"off", "perChunk"});
            o.inert.push_back(flag);
        } else if (flag == "--scatter") {
            o.scatter = next();
            expectOneOf(flag, o.scatter, {"shared", "direct"});
            o.kernelOnly.push_back(flag);
        } else if (flag == "--bin-path") {
            o.binPath = next();
            expectOneOf(flag, o.binPath, {"dense", "hash"});
            o.kernelOnly.push_back(flag);
        } else if (flag == "--bins") {
            o.bins = parseU32(flag, next());
            o.kernelOnly.push_back(flag);
        } else if (flag == "--distribution") {
            o.distribution = next();
            expectOneOf(flag, o.distribution, {"balanced", "one-hot", "skewed", "sparse"});
            o.kernelOnly.push_back(flag);
        } else {
            throw std::invalid_argument("unknown flag '" + flag + "'");
        }
    }
    if (!o.kernelOnly.empty() && o.workload != "kernel")
        throw std::invalid_argument("--scatter, --bin-path, --bins and --distribution require --workload kernel");
    return o;
}

// Sorted (weight, count) rows of w on the device; the caller's stream is the default stream.
void histogram(const std::vector<std::uint32_t>& w, std::vector<std::uint32_t>& values,
               std::vector<unsigned long long>& counts)
{
    const std::uint64_t n = w.size();
    values.clear();
    counts.clear();
    if (n == 0u)
        return;
    std::uint64_t scratch = 0u;
    if (gf_histogram_scratch_bytes(n, &scratch) != GF_OK)
        throw std::runtime_error("histogram scratch: " + lastError());
    void *d_w = nullptr, *d_scratch = nullptr, *d_rv = nullptr, *d_rc = nullptr, *d_small = nullptr;
    auto release = [&] {
        cudaFree(d_w);
        cudaFree(d_scratch);
        cudaFree(d_rv);
        cudaFree(d_rc);
        cudaFree(d_small);
    };
    try {
        cudaOrThrow(cudaMalloc(&d_w, n * sizeof(std::uint32_t)), "cudaMalloc");
        cudaOrThrow(cudaMalloc(&d_scratch, scratch), "cudaMalloc");
        cudaOrThrow(cudaMalloc(&d_rv, n * sizeof(std::uint32_t)), "cudaMalloc");
        cudaOrThrow(cudaMalloc(&d_rc, n * sizeof(unsigned long long)), "cudaMalloc");
        cudaOrThrow(cudaMalloc(&d_small, 2u * sizeof(std::uint32_t)), "cudaMalloc");
        cudaOrThrow(cudaMemcpy(d_w, w.data(), n * sizeof(std::uint32_t), cudaMemcpyHostToDevice), "H2D");
        cudaOrThrow(cudaMemset(d_small, 0, 2u * sizeof(std::uint32_t)), "cudaMemset");
        auto* small = static_cast<std::uint32_t*>(d_small);
        if (gf_histogram_u32(nullptr, static_cast<const std::uint32_t*>(d_w), n, d_scratch, scratch,
                             static_cast<std::uint32_t*>(d_rv), static_cast<unsigned long long*>(d_rc), small,
                             small + 1) != GF_OK)
            throw std::runtime_error("histogram: " + lastError());
        std::uint32_t h_small[2] = {0u, 0u};
        cudaOrThrow(cudaMemcpy(h_small, d_small, sizeof(h_small), cudaMemcpyDeviceToHost), "D2H");
        if (h_small[1] != 0u)
            throw std::runtime_error("histogram: device status " + std::to_string(h_small[1]));
        values.resize(h_small[0]);
        counts.resize(h_small[0]);
        cudaOrThrow(cudaMemcpy(values.data(), d_rv, h_small[0] * sizeof(std::uint32_t), cudaMemcpyDeviceToHost),
                    "D2H");
        cudaOrThrow(cudaMemcpy(counts.data(), d_rc, h_small[0] * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                    "D2H");
    } catch (...) {
        release();
        throw;
    }
    release();
}

int run(const Options& o)
{
    if (o.backend != "cuda")
        throw std::invalid_argument("--backend: this build runs on CUDA (sm_100a) only, got '" + o.backend + "'");
    const bool kernel = o.workload == "kernel";
    if (kernel) { // KernelAxes.hpp:169-214 checks, and this build's limits
        if (o.bins != 64u && o.bins != 1024u && o.bins != 4096u && o.bins != 65536u)
            throw std::invalid_argument("--bins: the kernel workload instantiates 64, 1024, 4096 and 65536 (got '" +
                                        std::to_string(o.bins) + "')");
        if (o.binPath == "hash" && o.scatter == "direct")
            throw std::invalid_argument("--scatter direct is the dense-path variant; the hash path always stages");
        if (o.distribution == "sparse" && o.bins < 1024u)
            throw std::invalid_argument("--distribution sparse requires --bins 1024 or larger");
        if (o.binPath == "dense" && o.bins > 4096u)
            throw std::invalid_argument("--bin-path dense supports at most 4096 bins here; use --bin-path hash above "
                                        "that");
    }
    for (const auto& f : o.inert)
        std::cerr << kName << ": note: " << f << " has no effect in this build\n";

    cudaOrThrow(cudaSetDevice(static_cast<int>(o.device)), "cudaSetDevice");
    if (o.deviceResident && gf_set_tuning("device_resident", 1) != GF_OK)
        throw std::runtime_error("device_resident: " + lastError());
    const bool wideChunk = !o.chunkSize || *o.chunkSize >= kLogicalTileWidth;
    gf_policy pol{};
    if (gf_device_policy(nullptr, o.particles, o.chunkSize.value_or(0u), o.liveParticles.value_or(0u),
                         o.tileSize.value_or(0u), wideChunk ? kAcceleratorLivePerChunk : 0u, 0u, 0u, &pol) != GF_OK)
        throw std::invalid_argument(lastError());
    const std::uint32_t C = pol.chunk_capacity, P = pol.live_particles, T = pol.tile_size;
    cudaDeviceProp prop{};
    cudaOrThrow(cudaGetDeviceProperties(&prop, static_cast<int>(o.device)), "cudaGetDeviceProperties");

    std::vector<std::uint32_t> weights(o.particles), capped(kernel ? 0u : o.particles);
    gf_flow_stats st{};
    if (kernel) {
        const int dist = o.distribution == "one-hot" ? GF_KDIST_ONEHOT
                         : o.distribution == "skewed" ? GF_KDIST_SKEWED
                         : o.distribution == "sparse" ? GF_KDIST_SPARSE
                                                      : GF_KDIST_BALANCED;
        const bool direct = o.scatter == "direct"; // the plain form's one-atomic-per-particle scatter
        if (gf_run_kernel_axes(o.seed, o.particles, o.bins, dist, direct ? GF_SCATTER_DIRECT : GF_SCATTER_SHARED,
                               o.binPath == "hash" ? 1 : 0, C, P, o.batchChunks, direct ? 0 : 1, weights.data(),
                               &st) != GF_OK)
            throw std::runtime_error(lastError());
    } else if (gf_run_particle_feedback(o.seed, o.particles, o.maxVisits, C, P, o.batchChunks, 1, GF_LAYOUT_SOA,
                                        weights.data(), capped.data(), &st) != GF_OK) {
        throw std::runtime_error(lastError());
    }
    std::vector<std::uint32_t> values;
    std::vector<unsigned long long> counts;
    histogram(weights, values, counts);
    std::uint64_t nCapped = 0u;
    for (const auto c : capped)
        nCapped += c != 0u ? 1u : 0u;

    std::cout << "# graphFlow_particle_feedback backend=cuda device=" << o.device << " device-name=" << prop.name
              << (kernel ? " workload=kernel" : "") << " particles=" << o.particles << " chunk-size=" << C
              << " live-particles=" << P << " tile-size=" << T << " batch-chunks=" << o.batchChunks
              << " seed=" << o.seed;
    if (kernel)
        std::cout << " scatter=" << o.scatter << " bin-path=" << o.binPath << " bins=" << o.bins
                  << " distribution=" << o.distribution << '\n';
    else
        std::cout << " max-visits=" << o.maxVisits << '\n';
    std::cout << "# pool-chunks=" << st.pool_chunks << " peak-live-chunks=" << st.peak_live_chunks
              << " peak-reserved-chunks=" << st.peak_reserved_chunks << '\n';
    std::cout << "# scheduler completed-batches=" << st.completed_batches << " partition-batches="
              << st.partition_batches << " kernel-launches=" << st.kernel_launches << " loop-iterations="
              << st.loop_iterations << " generated=" << st.generated << " sunk=" << st.sunk
              << " seconds=" << st.seconds << '\n';
    std::cout << "# weight,count\n";
    for (std::size_t i = 0; i < values.size(); ++i)
        std::cout << values[i] << ',' << counts[i] << '\n';
    if (o.particles != 0u && nCapped != 0u)
        std::cout << "# non-terminating " << nCapped << '\n';
    return EXIT_SUCCESS;
}

} // namespace

int main(int argc, char** argv)
{
    Options o;
    try {
        o = parse(argc, argv);
    } catch (const std::exception& e) {
        std::cerr << kName << ": " << e.what() << '\n';
        usage(std::cerr);
        return 2;
    }
    if (o.help) {
        usage(std::cout);
        return EXIT_SUCCESS;
    }
    try {
        return run(o);
    } catch (const std::invalid_argument& e) {
        std::cerr << kName << ": " << e.what() << '\n';
        usage(std::cerr);
        return 2;
    } catch (const std::exception& e) {
        std::cerr << kName << ": " << e.what() << '\n';
        return 1;
    }
}

// graphflow_b200_photon_scattering: a command-line drop-in for the reference example binary
// graphFlow_photon_scattering (examples/photon_scattering/main.cpp and PhotonCli.hpp). It takes the
// same flags (with their short aliases --N, --L, --sigmaS, --sigmaA, --cap, --C, --P, --T, --Q) and
// prints the same report: "# ..." provenance lines, "# event,count" with the transmitted,
// reflected, absorbed and capped counts, "# outcome,scatter-count,count" rows in (outcome,
// scatter count) order, "# terminal-sum,N" and "# inconsistent,K" (main.cpp:52-68 and
// PhotonScattering.hpp:132-156: a photon is consistent when it reached exactly one terminal
// event). The run is the reference example's analog model (absorption terminal, forward or
// isotropic scattering) in FP64, the reference's CUDA precision, through gf_run_photon on the
// current CUDA device; C, P and T the command line leaves out come from the device policy as in
// PhotonCli.hpp resolveOptions.
//
// --output-dir DIR writes the reference's run files (PhotonOutput.hpp:91-197 writeRunOutputs):
// metadata.csv, outcomes.csv, scatter_histogram.csv, exits.csv (one row per transmitted or
// reflected photon with its exit position and direction, 17 significant digits), traces.csv (the
// path trace vertices of the photons with id < --trace-photons, at most --trace-vertices each:
// source, every scatter with its outgoing direction, the terminal event) and trace_summary.csv
// (vertices kept and the truncation flag per traced id), through gf_run_photon_traced.
//
// Differences, by design: only --backend cuda runs. --exec fused (default) carries each photon
// through the same functors in one kernel and --exec flow runs the graph through the Flow; both
// give identical histories, traced or not. Pool, frame-cap, occupancy and per-chunk-schedule flags
// are checked as the reference does and reported inert on stderr; provenance keys of metadata.csv
// that name the reference's build (commit, alpaka pin, source directories) are written empty. At
// most 65535 scatters per photon (16-bit counter).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cli_common.hpp"
#include "graphflow_b200.h"

namespace {

using gfcli::cudaOrThrow;
using gfcli::expectOneOf;
using gfcli::lastError;
using gfcli::parseDouble;
using gfcli::parseU32;
using gfcli::parseU64;

constexpr const char* kName = "graphflow_b200_photon_scattering";
constexpr std::uint32_t kAcceleratorLivePerChunk = 8u; // DevicePolicy.hpp:53
constexpr std::uint32_t kLogicalTileWidth = 128u;
constexpr std::uint32_t kMaxScatters = 0xFFFFu;
const char* const kEventName[5] = {"scatter", "transmitted", "reflected", "absorbed", "capped"};

struct Options {
    bool help = false;
    std::string backend = "cpu";
    std::uint64_t photons = 0u;
    double thickness = 1.0, sigmaS = 0.0, sigmaA = 0.0;
    std::string mode = "forward";
    std::uint32_t maxScatters = 64u;
    std::uint64_t seed = 0u;
    std::optional<std::uint32_t> chunkSize, liveParticles, tileSize;
    std::uint32_t batchChunks = 1u;
    std::uint32_t device = 0u;
    std::string exec = "fused";
    bool deviceResident = false; // with --exec flow: the Flow run device-resident
    std::uint32_t frameCap = 8u; // LaunchPolicy.hpp:18 defaultFrameCap (inert here, recorded in metadata)
    std::optional<std::string> outputDir;
    std::uint32_t tracePhotons = 0u, traceVertices = 64u; // PhotonCli.hpp:46-47
    std::string command;
    std::vector<std::string> inert;
};

void usage(std::ostream& out)
{
    out << "usage: " << kName << " --backend cuda [--device D]\n"
           "                                        [--photons N] [--thickness L]\n"
           "                                        [--sigma-s S] [--sigma-a A]\n"
           "                                        [--mode forward|isotropic]\n"
           "                                        [--max-scatters M] [--seed S]\n"
           "                                        [--chunk-size C] [--live-particles P]\n"
           "                                        [--tile-size T] [--batch-chunks Q]\n"
           "                                        [--exec fused|flow] [--device-resident]\n"
           "       accepted for parity with graphFlow_photon_scattering, no effect here:\n"
           "       [--occupancy-target D] [--frame-cap F] [--pool-budget-bytes B]\n"
           "       [--pool-mode fixed|slotArena] [--slot-arena-budget BYTES]\n"
           "       [--chunk-kernel-schedule off|perChunk] [--chunk-queue-depth D]\n"
           "       [--chunk-latency-cap-us U]\n"
           "       [--output-dir DIR]   the reference's run files (metadata, outcomes, scatter histogram,\n"
           "                            exits, path traces)\n"
           "       [--trace-photons M] [--trace-vertices V]   trace ids < M, at most V vertices each\n"
           "                            (default 0 and 64)\n"
           "       defaults: L = 1, sigma-s = sigma-a = 0, forward, 64 scatters, seed 0; C, P and T from\n"
           "       the device policy; --exec fused (the Flow and the fused kernel give identical results).\n";
}

Options parse(int argc, char** argv)
{
    Options o;
    for (int i = 0; i < argc; ++i)
        o.command += (i ? " " : "") + std::string(argv[i]);
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
        } else if (flag == "--photons" || flag == "--N") {
            o.photons = parseU64(flag, next());
        } else if (flag == "--thickness" || flag == "--L") {
            o.thickness = parseDouble(flag, next());
        } else if (flag == "--sigma-s" || flag == "--sigmaS") {
            o.sigmaS = parseDouble(flag, next());
        } else if (flag == "--sigma-a" || flag == "--sigmaA") {
            o.sigmaA = parseDouble(flag, next());
        } else if (flag == "--mode") {
            o.mode = next();
            expectOneOf(flag, o.mode, {"forward", "isotropic"});
        } else if (flag == "--max-scatters" || flag == "--cap") {
            o.maxScatters = parseU32(flag, next(), true);
        } else if (flag == "--seed") {
            o.seed = parseU64(flag, next());
        } else if (flag == "--chunk-size" || flag == "--C") {
            o.chunkSize = parseU32(flag, next());
        } else if (flag == "--live-particles" || flag == "--P") {
            o.liveParticles = parseU32(flag, next());
        } else if (flag == "--tile-size" || flag == "--T") {
            o.tileSize = parseU32(flag, next());
        } else if (flag == "--batch-chunks" || flag == "--Q") {
            o.batchChunks = parseU32(flag, next());
        } else if (flag == "--device") {
            o.device = parseU32(flag, next(), true);
        } else if (flag == "--device-resident") {
            o.deviceResident = true;
        } else if (flag == "--exec") {
            o.exec = next();
            expectOneOf(flag, o.exec, {"fused", "flow"});
        } else if (flag == "--frame-cap") {
            o.frameCap = parseU32(flag, next());
            o.inert.push_back(flag);
        } else if (flag == "--chunk-queue-depth") {
            parseU32(flag, next());
            o.inert.push_back(flag);
        } else if (flag == "--occupancy-target" || flag == "--chunk-latency-cap-us") {
            parseU32(flag, next(), true);
            o.inert.push_back(flag);
        } else if (flag == "--pool-budget-bytes") {
            if (parseU64(flag, next()) == 0u)
                throw std::invalid_argument(flag + ": value must be non-zero");
            o.inert.push_back(flag);
        } else if (flag == "--slot-arena-budget") {
            parseU64(flag, next());
            o.inert.push_back(flag);
        } else if (flag == "--pool-mode") {
            expectOneOf(flag, next(), {"fixed", "slotArena"});
            o.inert.push_back(flag);
        } else if (flag == "--chunk-kernel-schedule") {
            expectOneOf(flag, next(), {"off", "perChunk"});
            o.inert.push_back(flag);
        } else if (flag == "--output-dir") {
            o.outputDir = next();
            if (o.outputDir->empty())
                throw std::invalid_argument("--output-dir: value must not be empty");
        } else if (flag == "--trace-photons") {
            o.tracePhotons = parseU32(flag, next(), true);
        } else if (flag == "--trace-vertices") {
            o.traceVertices = parseU32(flag, next(), true);
        } else {
            throw std::invalid_argument("unknown argument '" + flag + "'");
        }
    }
    if (o.deviceResident && o.exec != "flow")
        throw std::invalid_argument("--device-resident requires --exec flow");
    return o;
}

int run(const Options& o)
{
    if (o.backend != "cuda")
        throw std::invalid_argument("--backend: this build runs on CUDA (sm_100a) only, got '" + o.backend + "'");
    if (!(o.thickness > 0.0))
        throw std::invalid_argument("--thickness: must be positive");
    if (o.sigmaS < 0.0 || o.sigmaA < 0.0)
        throw std::invalid_argument("--sigma-s / --sigma-a: must not be negative");
    if (o.maxScatters > kMaxScatters)
        throw std::invalid_argument("--max-scatters: at most 65535 in this build");
    for (const auto& f : o.inert)
        std::cerr << kName << ": note: " << f << " has no effect in this build\n";

    cudaOrThrow(cudaSetDevice(static_cast<int>(o.device)), "cudaSetDevice");
    if (o.deviceResident && gf_set_tuning("device_resident", 1) != GF_OK)
        throw std::runtime_error("device_resident: " + lastError());
    cudaDeviceProp prop{};
    cudaOrThrow(cudaGetDeviceProperties(&prop, static_cast<int>(o.device)), "cudaGetDeviceProperties");
    const bool wideChunk = !o.chunkSize || *o.chunkSize >= kLogicalTileWidth;
    gf_policy pol{};
    if (gf_device_policy(nullptr, o.photons, o.chunkSize.value_or(0u), o.liveParticles.value_or(0u),
                         o.tileSize.value_or(0u), wideChunk ? kAcceleratorLivePerChunk : 0u, 0u, 0u, &pol) != GF_OK)
        throw std::invalid_argument(lastError());

    gf_photon_params p{};
    p.thickness = o.thickness;
    p.sigma_s = o.sigmaS;
    p.sigma_a = o.sigmaA;
    p.max_scatters = o.maxScatters;
    p.model = GF_PHOTON_ANALOG;
    p.isotropic = o.mode == "isotropic" ? 1 : 0;
    p.fp64 = 1;
    const std::size_t m = o.photons ? o.photons : 1u;
    std::vector<std::uint32_t> event(m), scatters(m);
    std::vector<double> position(o.outputDir ? 3u * m : 0u), direction(o.outputDir ? 3u * m : 0u);
    std::vector<std::uint64_t> eventCounts(5, 0u);
    gf_flow_stats st{};
    // path trace of ids < M (PhotonScattering.hpp:49-57: M = min(N, --trace-photons))
    const std::uint64_t traceIds = std::min<std::uint64_t>(o.photons, o.tracePhotons);
    std::vector<gf_trace_vertex> traceVertices(traceIds * o.traceVertices);
    std::vector<std::uint32_t> traceCounts(traceIds), traceTruncated(traceIds);
    if (gf_run_photon_traced(o.seed, 0u, o.photons, &p, o.exec == "flow" ? GF_EXEC_FLOW : GF_EXEC_FUSED,
                             pol.chunk_capacity, pol.live_particles, o.batchChunks, event.data(), scatters.data(),
                             nullptr, nullptr, o.outputDir ? position.data() : nullptr,
                             o.outputDir ? direction.data() : nullptr, nullptr, nullptr, eventCounts.data(), &st,
                             o.tracePhotons, o.traceVertices, traceVertices.data(), traceCounts.data(),
                             traceTruncated.data()) != GF_OK)
        throw std::runtime_error(lastError());
    std::uint64_t traceTruncatedIds = 0u;
    for (const std::uint32_t t : traceTruncated)
        traceTruncatedIds += t != 0u;

    // outcome histogram over the delivered photons (PhotonScattering.hpp:132-156)
    std::map<std::pair<std::uint32_t, std::uint32_t>, std::uint64_t> rows;
    std::uint64_t counts[5] = {0u, 0u, 0u, 0u, 0u}, terminated = 0u, inconsistent = 0u;
    for (std::uint64_t id = 0; id < o.photons; ++id) {
        const std::uint32_t e = event[id];
        if (e == 0u || e > 4u) {
            ++inconsistent;
            continue;
        }
        ++terminated;
        ++counts[e];
        ++rows[{e, scatters[id]}];
    }

    std::cout << "# graphFlow_photon_scattering backend=cuda device=" << o.device << " device-name=" << prop.name
              << " photons=" << o.photons << " thickness=" << o.thickness << " sigma-s=" << o.sigmaS
              << " sigma-a=" << o.sigmaA << " mode=" << o.mode << " max-scatters=" << o.maxScatters
              << " seed=" << o.seed << " chunk-size=" << pol.chunk_capacity
              << " live-particles=" << (o.photons ? pol.live_particles : 1u) << " tile-size=" << pol.tile_size
              << " batch-chunks=" << o.batchChunks << " exec=" << o.exec << '\n';
    std::cout << "# units length=1 coefficient=1/length\n";
    std::cout << "# pool-chunks=" << st.pool_chunks << " peak-live-chunks=" << st.peak_live_chunks
              << " peak-reserved-chunks=" << st.peak_reserved_chunks << '\n';
    std::cout << "# scheduler completed-batches=" << st.completed_batches << " partition-batches="
              << st.partition_batches << " kernel-launches=" << st.kernel_launches << " loop-iterations="
              << st.loop_iterations << " seconds=" << st.seconds << '\n';
    std::cout << "# event,count\n";
    for (const std::uint32_t e : {1u, 2u, 3u, 4u})
        std::cout << kEventName[e] << ',' << counts[e] << '\n';
    std::cout << "# outcome,scatter-count,count\n";
    for (const auto& [key, count] : rows)
        std::cout << kEventName[key.first] << ',' << key.second << ',' << count << '\n';
    std::cout << "# terminal-sum," << terminated << '\n';
    std::cout << "# inconsistent," << inconsistent << '\n';

    if (o.outputDir) {
        const std::filesystem::path dir(*o.outputDir);
        std::filesystem::create_directories(dir);
        std::ofstream meta(dir / "metadata.csv"), outcomes(dir / "outcomes.csv"), hist(dir / "scatter_histogram.csv"),
            exits(dir / "exits.csv"), traces(dir / "traces.csv"), summary(dir / "trace_summary.csv");
        if (!meta || !outcomes || !hist || !exits || !traces || !summary)
            throw std::runtime_error("cannot create the output files in '" + *o.outputDir + "'");
        outcomes << "event,count\n";
        for (const std::uint32_t e : {1u, 2u, 3u, 4u})
            outcomes << kEventName[e] << ',' << counts[e] << '\n';
        hist << "event,scatter_count,count\n";
        for (const auto& [key, count] : rows)
            hist << kEventName[key.first] << ',' << key.second << ',' << count << '\n';
        exits << "id,event,scatter_count,x,y,z,ux,uy,uz,cos_theta,phi_rad,transverse_x,transverse_y\n";
        exits << std::setprecision(17);
        for (std::uint64_t id = 0; id < o.photons; ++id) {
            if (event[id] != 1u && event[id] != 2u)
                continue;
            const double* x = &position[3u * id];
            const double* u = &direction[3u * id];
            exits << id << ',' << kEventName[event[id]] << ',' << scatters[id] << ',' << x[0] << ',' << x[1] << ','
                  << x[2] << ',' << u[0] << ',' << u[1] << ',' << u[2] << ',' << u[2] << ',' << std::atan2(u[1], u[0])
                  << ',' << x[0] << ',' << x[1] << '\n';
        }
        // PhotonOutput.hpp:56-75 traceName, :131-146 the trace rows
        static const char* const kTraceName[6] = {"source",   "scatter",  "transmitted",
                                                  "reflected", "absorbed", "capped"};
        traces << "id,step,kind,scatter_count,x,y,z,ux,uy,uz\n";
        traces << std::setprecision(17);
        summary << "id,vertices,truncated\n";
        for (std::uint64_t id = 0; id < traceIds; ++id) {
            summary << id << ',' << traceCounts[id] << ',' << (traceTruncated[id] != 0u ? 1 : 0) << '\n';
            for (std::uint32_t step = 0; step < traceCounts[id]; ++step) {
                const gf_trace_vertex& v = traceVertices[id * o.traceVertices + step];
                traces << id << ',' << step << ',' << (v.kind < 6u ? kTraceName[v.kind] : "unknown") << ','
                       << v.scatter_count << ',' << v.position[0] << ',' << v.position[1] << ',' << v.position[2]
                       << ',' << v.direction[0] << ',' << v.direction[1] << ',' << v.direction[2] << '\n';
            }
        }
        auto quote = [](const std::string& v) {
            std::string q = "\"";
            for (const char c : v)
                q += c == '"' ? std::string("\"\"") : std::string(1, c);
            return q + "\"";
        };
        auto kv = [&](const char* key, const std::string& value) { meta << key << ',' << quote(value) << '\n'; };
        auto kn = [&](const char* key, auto value) { kv(key, std::to_string(value)); };
        meta << "key,value\n";
        kv("schema_version", "1");
        kv("graphflow_commit", "");
        kv("alpaka_pin", "");
        kv("graphflow_source_dir", "");
        kv("alpaka_source_dir", "");
        kv("backend", "cuda");
        kn("device_index", o.device);
        kv("device_name", prop.name);
        kv("device_api", "cuda");
        kn("multiprocessor_count", prop.multiProcessorCount);
        kn("warp_size", prop.warpSize);
        kn("global_mem_bytes", static_cast<std::uint64_t>(prop.totalGlobalMem));
        kv("command", o.command);
        kv("units", "length=1 coefficient=1/length angle=rad");
        kn("photons", o.photons);
        kn("thickness", o.thickness);
        kn("sigma_s", o.sigmaS);
        kn("sigma_a", o.sigmaA);
        kn("sigma_t", o.sigmaS + o.sigmaA);
        kv("mode", o.mode);
        kn("max_scatters", o.maxScatters);
        kn("seed", o.seed);
        kn("chunk_size", pol.chunk_capacity);
        kn("live_particles", o.photons ? pol.live_particles : 1u);
        kn("tile_size", pol.tile_size);
        kn("batch_chunks", o.batchChunks);
        kn("frame_cap", o.frameCap);
        kn("pool_chunks", st.pool_chunks);
        kn("peak_live_chunks", st.peak_live_chunks);
        kn("peak_reserved_chunks", st.peak_reserved_chunks);
        kv("scheduler_stats", "completed-batches=" + std::to_string(st.completed_batches) +
                                  " partition-batches=" + std::to_string(st.partition_batches) +
                                  " kernel-launches=" + std::to_string(st.kernel_launches));
        kn("count_terminated", terminated);
        kn("count_inconsistent", inconsistent);
        kn("count_transmitted", counts[1]);
        kn("count_reflected", counts[2]);
        kn("count_absorbed", counts[3]);
        kn("count_capped", counts[4]);
        kn("trace_enabled", o.tracePhotons != 0u ? 1 : 0);
        kn("trace_photons", o.tracePhotons);
        kn("trace_vertices", o.traceVertices);
        kn("trace_ids", traceIds);
        kn("trace_truncated_ids", traceTruncatedIds);
        kn("detector_distance", o.thickness);
        kn("detector_half_width", 2.0 * o.thickness);
        std::cout << "# output-dir=" << *o.outputDir << '\n';
    }
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

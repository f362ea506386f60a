// photon_scattering transform bodies on the graphflow_b200 C++ front end.
//
// Topology (examples/photon_scattering/PhotonScattering.hpp:84-102 in graphFlow):
//   source -> propose flight (transform) -> advance and route (partition, 5 bins)
//          -> scatter (transform) -> propose flight; transmitted/reflected/absorbed/capped -> terminal
// Node keys fix the stream purposes: flight 2, route 4 (+1 updater), scatter 6.
//
// Two models share that graph:
//   * analog (the reference example, PhotonFunctors.hpp:35-415): absorption is a terminal event,
//     forward or isotropic scattering, no weight;
//   * weighted (the FP32 Monte Carlo sweep): Henyey-Greenstein scattering with anisotropy g,
//     implicit capture w *= mu_s / mu_t at every collision, Russian roulette below a weight
//     threshold (survive with probability p, weight / p), loop until exit; exit weights are
//     histogrammed by exit |cos theta| for reflection and transmission. Sampling and direction
//     update are the published MCML forms (Wang, Jacques, Zheng 1995).
// Draws per stream position: flight stage d0 = path length, d1 = collision kind (analog) or
// roulette (weighted); scatter stage d0 = cos theta, d1 = azimuth.
#pragma once

#include <cstdint>

#include "graphflow/flow.cuh"

namespace graphflow::photon {

enum class Event : std::uint32_t { scatter = 0u, transmitted = 1u, reflected = 2u, absorbed = 3u, capped = 4u };
inline constexpr std::uint32_t eventBins = 5u;

template <typename T>
struct Vec3T {
    T x, y, z;
};

template <typename T>
struct ProposalT {
    Event event;
    T distance;
    T nextWeight; // weighted model: weight after this event
    std::uint32_t valid;
};

template <typename T>
struct PhotonT {
    std::uint64_t id;
    Vec3T<T> position;
    Vec3T<T> direction;
    T weight;
    std::uint32_t scatterCount;
    ProposalT<T> proposal;
};

template <typename T>
struct SlabT {
    T thickness, sigmaS, sigmaA;
};

template <typename T>
struct WeightedT {
    T g, rouletteThreshold, rouletteSurvival;
};

// Terminal record of one history (PhotonTypes.hpp:186-196 + weight).
template <typename T>
struct TerminalT {
    std::uint32_t event;
    std::uint32_t scatterCount;
    T weight;
    T cosExit;
    Vec3T<T> position;
    Vec3T<T> direction; // at the terminal event (the exit direction for the two exits)
};

// Path trace vertex kinds (PhotonTypes.hpp:189-197): the source, each scatter, then the terminal
// event as Event + 1.
enum class TraceKind : std::uint32_t {
    source = 0u,
    scatter = 1u,
    transmitted = 2u,
    reflected = 3u,
    absorbed = 4u,
    capped = 5u
};

template <typename T>
struct TraceVertexT {
    TraceKind kind;
    std::uint32_t scatterCount; // completed scatters, this one included
    Vec3T<T> position;
    Vec3T<T> direction; // outgoing
};

// Trace writer of untraced runs (PhotonFunctors.hpp:188-199): the functors' default, so their
// kernels carry no trace code at all.
template <typename T>
struct NoTraceT {
    __device__ void record(std::uint64_t, TraceKind, std::uint32_t, const Vec3T<T>&, const Vec3T<T>&) const {}
};

// Bounded path trace (PhotonFunctors.hpp:201-234): photons with id < limit own maxVertices
// consecutive vertex slots; a vertex past the bound sets the id's truncation flag instead and
// leaves the history alone. A photon's events run one after another on one thread at a time, in
// the Flow and in the fused kernel alike, so its counter needs no atomic.
template <typename T>
struct TraceT {
    TraceVertexT<T>* vertices = nullptr;
    std::uint32_t* counts = nullptr;
    std::uint32_t* truncated = nullptr;
    std::uint32_t maxVertices = 0u;
    std::uint64_t limit = 0u;
    __device__ void record(std::uint64_t id, TraceKind kind, std::uint32_t scatterCount, const Vec3T<T>& position,
                           const Vec3T<T>& direction) const
    {
        if (id >= limit)
            return;
        const std::uint32_t index = counts[id];
        if (index >= maxVertices) {
            truncated[id] = 1u;
            return;
        }
        vertices[id * maxVertices + index] = TraceVertexT<T>{kind, scatterCount, position, direction};
        counts[id] = index + 1u;
    }
};

template <typename T>
__device__ inline T dlog(T x)
{
    if constexpr (sizeof(T) == 4)
        return logf(x);
    else
        return log(x);
}

// PhotonFunctors.hpp:35-52 faceHit + :55-59 faceFirst (equality belongs to the face).
template <typename T>
__device__ inline bool faceHit(const SlabT<T>& s, const PhotonT<T>& p, T& dist, Event& ev)
{
    if (p.direction.z > T(0)) {
        dist = (s.thickness - p.position.z) / p.direction.z;
        ev = Event::transmitted;
        return true;
    }
    if (p.direction.z < T(0)) {
        dist = -p.position.z / p.direction.z;
        ev = Event::reflected;
        return true;
    }
    return false;
}

template <typename T, typename TTrace = NoTraceT<T>>
struct GeneratePhotonT {
    TTrace trace;
    __device__ PhotonT<T> operator()(const Acc&, std::uint64_t id) const
    {
        PhotonT<T> p{};
        p.id = id;
        p.position = {T(0), T(0), T(0)};
        p.direction = {T(0), T(0), T(1)};
        p.weight = T(1);
        p.scatterCount = 0u;
        p.proposal = ProposalT<T>{Event::absorbed, T(0), T(1), 0u};
        trace.record(id, TraceKind::source, 0u, p.position, p.direction);
        return p;
    }
};

// PhotonFunctors.hpp:270-288 ProposeFlight + :73-123 resolveFlight (analog model).
template <typename T>
struct ProposeFlightT {
    SlabT<T> slab;
    std::uint32_t maxScatters;
    __device__ void operator()(const Acc&, rng::Engine& e, Status& st, PhotonT<T>& p) const
    {
        const T flight = T(1) - rng::uniform<T>(e);
        const T kind = rng::uniform<T>(e);
        const T total = slab.sigmaS + slab.sigmaA;
        const T sampled = total > T(0) ? -dlog(flight) / total : T(0);
        T fd = T(0);
        Event fe = Event::absorbed;
        const bool reach = faceHit(slab, p, fd, fe);
        ProposalT<T> pr{Event::absorbed, T(0), p.weight, 0u};
        if (total == T(0)) {
            if (reach) {
                pr.event = fe;
                pr.distance = fd;
                pr.valid = 1u;
            }
        } else if (reach && fd <= sampled) {
            pr.event = fe;
            pr.distance = fd;
            pr.valid = 1u;
        } else {
            const bool scatters = kind < slab.sigmaS / total;
            pr.distance = sampled;
            pr.event = !scatters ? Event::absorbed : (p.scatterCount >= maxScatters ? Event::capped : Event::scatter);
            pr.valid = 1u;
        }
        p.proposal = pr;
        if (!pr.valid)
            st.set(StatusCode::invalid);
    }
};

// Weighted model: flight draw d0, roulette draw d1; the proposal carries the next weight.
template <typename T>
struct ProposeWeightedT {
    SlabT<T> slab;
    WeightedT<T> w;
    std::uint32_t maxScatters;
    __device__ void operator()(const Acc&, rng::Engine& e, Status& st, PhotonT<T>& p) const
    {
        const T mt = slab.sigmaS + slab.sigmaA;
        const T s = -dlog(T(1) - rng::uniform<T>(e)) / mt;
        const T roulette = rng::uniform<T>(e);
        T fd = T(0);
        Event fe = Event::absorbed;
        const bool reach = faceHit(slab, p, fd, fe);
        ProposalT<T> pr{Event::absorbed, s, p.weight, 1u};
        if (reach && fd <= s) {
            pr.event = fe;
            pr.distance = fd;
        } else {
            T nw = p.weight * (slab.sigmaS / mt);
            bool alive = true;
            if (nw < w.rouletteThreshold) {
                if (roulette < w.rouletteSurvival)
                    nw = nw / w.rouletteSurvival;
                else
                    alive = false;
            }
            pr.nextWeight = nw;
            pr.event = !alive ? Event::absorbed : (p.scatterCount >= maxScatters ? Event::capped : Event::scatter);
        }
        if (!(mt > T(0)))
            st.set(StatusCode::invalid);
        p.proposal = pr;
    }
};

// PhotonFunctors.hpp:292-314 ClassifyEvent.
template <typename T>
struct ClassifyEventT {
    static constexpr std::uint32_t maxBins = eventBins;
    __device__ Event operator()(const Acc&, Status& st, const PhotonT<T>& p) const
    {
        if (!p.proposal.valid || static_cast<std::uint32_t>(p.proposal.event) >= maxBins) {
            st.set(StatusCode::invalid);
            return Event::absorbed;
        }
        return p.proposal.event;
    }
};

// PhotonFunctors.hpp:130-170 applyEvent / :319-333 AdvanceToEvent (+ the weight update).
template <typename T>
struct AdvanceToEventT {
    SlabT<T> slab;
    __device__ UpdateResult operator()(const Acc&, Event ev, PhotonT<T>& p) const
    {
        if (!p.proposal.valid || ev != p.proposal.event)
            return UpdateResult::invalid;
        const T d = p.proposal.distance;
        p.position.x += d * p.direction.x;
        p.position.y += d * p.direction.y;
        switch (ev) {
        case Event::transmitted:
            if (p.direction.z <= T(0))
                return UpdateResult::invalid;
            p.position.z = slab.thickness;
            break;
        case Event::reflected:
            if (p.direction.z >= T(0))
                return UpdateResult::invalid;
            p.position.z = T(0);
            break;
        default:
            p.position.z += d * p.direction.z;
            p.weight = p.proposal.nextWeight;
            break;
        }
        return UpdateResult::success;
    }
};

// PhotonFunctors.hpp:172-186 isotropicDirection, :338-372 Scatter (analog model).
template <typename T, typename TTrace = NoTraceT<T>>
struct ScatterT {
    bool isotropic;
    TTrace trace;
    __device__ void operator()(const Acc&, rng::Engine& e, Status& st, PhotonT<T>& p) const
    {
        if (!p.proposal.valid || p.proposal.event != Event::scatter) {
            st.set(StatusCode::invalid);
            return;
        }
        if (isotropic) {
            const T pi = T(3.14159265358979323846);
            const T mu = T(2) * rng::uniform<T>(e) - T(1);
            const T phi = T(2) * pi * rng::uniform<T>(e);
            const T tr = sqrt(fmax(T(0), T(1) - mu * mu));
            p.direction = {tr * cos(phi), tr * sin(phi), mu};
        }
        if (p.scatterCount == 0xFFFFFFFFu) {
            st.set(StatusCode::overflow);
            return;
        }
        trace.record(p.id, TraceKind::scatter, p.scatterCount + 1u, p.position, p.direction);
        ++p.scatterCount;
    }
};

// Henyey-Greenstein scattering with the MCML direction update.
template <typename T, typename TTrace = NoTraceT<T>>
struct ScatterHGT {
    T g;
    TTrace trace;
    __device__ void operator()(const Acc&, rng::Engine& e, Status& st, PhotonT<T>& p) const
    {
        if (!p.proposal.valid || p.proposal.event != Event::scatter) {
            st.set(StatusCode::invalid);
            return;
        }
        const T xi = rng::uniform<T>(e);
        const T phi = T(2) * T(3.14159265358979323846) * rng::uniform<T>(e);
        T ct;
        if (g == T(0)) {
            ct = T(2) * xi - T(1);
        } else {
            const T t = (T(1) - g * g) / (T(1) - g + T(2) * g * xi);
            ct = (T(1) + g * g - t * t) / (T(2) * g);
            ct = ct < T(-1) ? T(-1) : (ct > T(1) ? T(1) : ct);
        }
        const T st2 = sqrt(fmax(T(0), T(1) - ct * ct));
        const T cp = cos(phi), sp = sin(phi);
        Vec3T<T>& u = p.direction;
        const T lim = sizeof(T) == 4 ? T(1) - T(1e-6) : T(1) - T(1e-12);
        if (fabs(u.z) > lim) {
            u = {st2 * cp, st2 * sp, u.z >= T(0) ? ct : -ct};
        } else {
            const T tmp = sqrt(T(1) - u.z * u.z);
            const T nx = st2 * (u.x * u.z * cp - u.y * sp) / tmp + u.x * ct;
            const T ny = st2 * (u.y * u.z * cp + u.x * sp) / tmp + u.y * ct;
            const T nz = -st2 * cp * tmp + u.z * ct;
            u = {nx, ny, nz};
        }
        trace.record(p.id, TraceKind::scatter, p.scatterCount + 1u, p.position, p.direction);
        ++p.scatterCount;
    }
};

// PhotonFunctors.hpp:377-415 RecordTerminal (+ exit-weight histograms of the weighted model).
template <typename T, typename TTrace = NoTraceT<T>>
struct RecordTerminalT {
    TerminalT<T>* records;
    std::uint32_t* visits;
    T* reflHist;   // may be null
    T* transHist;  // may be null
    std::uint32_t histBins;
    unsigned long long* eventCounts; // [5], may be null
    TTrace trace;                    // also the source's, so both execution forms trace alike
    __device__ void operator()(const Acc&, Status& st, const PhotonT<T>& p) const
    {
        const std::uint32_t ev = static_cast<std::uint32_t>(p.proposal.event);
        if (!p.proposal.valid || ev == 0u || ev >= eventBins) {
            st.set(StatusCode::invalid);
            return;
        }
        const T c = fabs(p.direction.z);
        if (records != nullptr)
            records[p.id] = TerminalT<T>{ev, p.scatterCount, p.weight, c, p.position, p.direction};
        trace.record(p.id, static_cast<TraceKind>(ev + 1u), p.scatterCount, p.position, p.direction);
        if (visits != nullptr && atomicAdd(&visits[p.id], 1u) != 0u)
            st.set(StatusCode::invalid);
        if (eventCounts != nullptr)
            atomicAdd(&eventCounts[ev], 1ull);
        if (histBins != 0u && (ev == 1u || ev == 2u)) {
            std::uint32_t b = static_cast<std::uint32_t>(c * T(histBins));
            b = b >= histBins ? histBins - 1u : b;
            atomicAdd(ev == 1u ? &transHist[b] : &reflHist[b], p.weight);
        }
    }
};

// The walks of one thread's photons (grid-stride over [0, n)).
template <typename T, typename TPropose, typename TScatter, typename TTrace>
__device__ void transport_walks(const TPropose& propose, const AdvanceToEventT<T>& advance, const TScatter& scatter,
                                const RecordTerminalT<T, TTrace>& terminal, std::uint64_t seedMixed,
                                std::uint64_t firstId, std::uint64_t n, std::uint32_t* status)
{
    const Acc acc{};
    Status st(status);
    const std::uint64_t stride = (std::uint64_t)gridDim.x * blockDim.x;
    std::uint64_t i = (std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const GeneratePhotonT<T, TTrace> generate{terminal.trace};
    PhotonT<T> p = generate(acc, firstId + i);
    std::uint32_t scatters = 0;
    // One event per iteration; a lane whose photon ends (or reaches 0x10001 scatters) starts its
    // next photon at once, so a warp stays full instead of waiting for its longest walk. Every
    // photon's draws are keyed by its own id and counters, so results do not depend on the order.
    for (;;) {
        rng::Engine ef = rng::engineFor(seedMixed, p, rng::streamPurposeForNode(1));
        propose(acc, ef, st, p);
        bool done;
        if (advance(acc, p.proposal.event, p) != UpdateResult::success) {
            st.set(StatusCode::invalid);
            done = true;
        } else if (p.proposal.event != Event::scatter) {
            terminal(acc, st, p);
            done = true;
        } else {
            rng::Engine es = rng::engineFor(seedMixed, p, rng::streamPurposeForNode(3));
            scatter(acc, es, st, p);
            done = ++scatters > 0x10000u;
        }
        if (done) {
            i += stride;
            if (i >= n)
                break;
            p = generate(acc, firstId + i);
            scatters = 0;
        }
    }
}

// Fused transport: a thread carries photons through propose -> advance -> scatter until their
// terminal events (transport_walks), calling the very functors the graph runs at the same stream
// positions, so a history is identical to the one the Flow produces.
template <typename T, typename TPropose, typename TScatter, typename TTrace>
__global__ void __launch_bounds__(256) transport_kernel(TPropose propose, AdvanceToEventT<T> advance, TScatter scatter,
                                                        RecordTerminalT<T, TTrace> terminal, std::uint64_t seedMixed,
                                                        std::uint64_t firstId, std::uint64_t n, std::uint32_t* status)
{
    // The event counts and exit histograms of this CTA's photons accumulate in shared memory
    // (every photon ends in one of two events, so device atomics per photon would queue on two
    // words) and are added to the device arrays once at the end.
    constexpr std::uint32_t kLocalHistBins = 1024u;
    __shared__ T s_hist[2][kLocalHistBins];
    __shared__ unsigned long long s_counts[eventBins];
    const bool localHist = terminal.histBins != 0u && terminal.histBins <= kLocalHistBins &&
                           terminal.transHist != nullptr && terminal.reflHist != nullptr;
    for (std::uint32_t k = threadIdx.x; k < 2u * kLocalHistBins; k += blockDim.x)
        s_hist[k / kLocalHistBins][k % kLocalHistBins] = T(0);
    for (std::uint32_t k = threadIdx.x; k < eventBins; k += blockDim.x)
        s_counts[k] = 0ull;
    __syncthreads();
    RecordTerminalT<T, TTrace> local = terminal;
    if (localHist) {
        local.transHist = s_hist[0];
        local.reflHist = s_hist[1];
    }
    if (terminal.eventCounts != nullptr)
        local.eventCounts = s_counts;
    transport_walks(propose, advance, scatter, local, seedMixed, firstId, n, status);
    __syncthreads();
    if (terminal.eventCounts != nullptr)
        for (std::uint32_t k = threadIdx.x; k < eventBins; k += blockDim.x)
            if (s_counts[k] != 0ull)
                atomicAdd(&terminal.eventCounts[k], s_counts[k]);
    if (localHist)
        for (std::uint32_t k = threadIdx.x; k < 2u * terminal.histBins; k += blockDim.x) {
            const std::uint32_t h = k / terminal.histBins, bin = k % terminal.histBins;
            if (s_hist[h][bin] != T(0))
                atomicAdd(h == 0u ? &terminal.transHist[bin] : &terminal.reflHist[bin], s_hist[h][bin]);
        }
}

} // namespace graphflow::photon

template <typename T>
struct graphflow::SoAFields<graphflow::photon::PhotonT<T>> {
    static constexpr std::size_t count = 6;
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        f(p.id);
        f(p.position);
        f(p.direction);
        f(p.weight);
        f(p.scatterCount);
        f(p.proposal);
    }
};

namespace graphflow::photon {

// Builds and runs the photon graph (PhotonScattering.hpp:37-181).
template <typename T, typename TStorage, typename TPropose, typename TScatter, typename TTrace>
SchedulerStats runPhotonFlow(cuda::Device device, std::uint64_t n, TPropose propose, SlabT<T> slab, TScatter scatter,
                             RecordTerminalT<T, TTrace> terminal, Tuning tuning)
{
    Flow<PhotonT<T>, cuda::Device, TStorage> flow{device};
    auto source = flow.source("generate", GeneratePhotonT<T, TTrace>{terminal.trace});
    auto flight = flow.transform("propose flight", propose);
    auto route = flow.partition("advance and route", ClassifyEventT<T>{}, AdvanceToEventT<T>{slab});
    auto scat = flow.transform("scatter", scatter);
    auto term = flow.sink("terminal", terminal);
    flow.connect(source, flight);
    flow.connect(flight, route);
    flow.connect(route.template out<Event::scatter>(), scat);
    flow.connect(scat, flight);
    flow.connect(route.template out<Event::transmitted>(), term);
    flow.connect(route.template out<Event::reflected>(), term);
    flow.connect(route.template out<Event::absorbed>(), term);
    flow.connect(route.template out<Event::capped>(), term);
    flow.configure(tuning);
    return flow.run(source, n);
}

} // namespace graphflow::photon

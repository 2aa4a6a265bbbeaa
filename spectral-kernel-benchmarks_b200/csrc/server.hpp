// Continuous-batching request loop for flux evaluations of mixed grid sizes.
//
// Each size class (n, Nz, targets, precision) owns one or more slots: a flux
// pipeline built for `maxBatch` ensemble members, its own CUDA stream and
// device staging.  Requests wait in their class's queue; a worker thread
// hands every free slot the oldest queued requests of its class (up to
// maxBatch) as soon as the slot's previous batch has finished, so requests
// that arrive while others run join the next batch, and slots of different
// classes (or several slots of one class) run concurrently on the GPU.
// Spectral states can be made resident on the device once and referenced by
// later requests.  Admission is by HBM footprint: slots are created while they
// fit the budget, and a resident state is admitted only if it fits what is
// left.  Every member of a batch is computed independently, so a request's
// result does not depend on which requests share its batch.

#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "flux.hpp"

namespace skb {

struct ServerClass {
    std::uint64_t n = 0, nz = 0, targets = 4, maxBatch = 1;
    FluxMode mode = FluxMode::fp64_plain;
};

struct ServerStats {
    std::uint64_t submitted = 0, completed = 0, batches = 0, slots = 0, residentStates = 0;
    std::uint64_t slotBytes = 0, stateBytes = 0, budgetBytes = 0;
};

class Server {
public:
    Server(const std::vector<ServerClass>& classes, std::uint64_t hbmBudget, int maxSlotsPerClass);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Element counts (complex) of one member's modal input / output.
    std::uint64_t inputElements(int cls) const;
    std::uint64_t outputElements(int cls) const;

    // Host FP64 complex input and output; returns a ticket.
    std::uint64_t submit(int cls, const double* input, double* output);
    // Input from a resident state.
    std::uint64_t submitState(std::int64_t state, double* output);
    std::int64_t loadState(int cls, const double* input);
    void releaseState(std::int64_t state);
    // Wait up to timeoutSeconds; returns true when finished and fills the
    // latency (submit -> result in host memory) in milliseconds.
    bool wait(std::uint64_t ticket, double timeoutSeconds, double* latencyMs);
    // While held, queued requests wait and no new batch starts (running
    // batches finish); releasing lets a burst that queued meanwhile be batched.
    void hold(bool held);
    ServerStats stats();

private:
    using Clock = std::chrono::steady_clock;
    struct Request {
        std::uint64_t ticket = 0;
        int cls = 0;
        const double* input = nullptr;
        std::int64_t state = -1;
        double* output = nullptr;
        Clock::time_point submitted, finished;
        bool done = false;
        int status = 0;
        std::string error;
    };
    struct Slot {
        int cls = 0;
        std::unique_ptr<FluxPipeline> flux;
        cudaStream_t stream = nullptr;
        cudaEvent_t event = nullptr;
        DeviceBuffer in, out, stage;  // pipeline-precision I/O and FP64 staging
        std::vector<std::shared_ptr<Request>> batch;
        bool busy = false;
    };
    struct State {
        int cls = 0;
        DeviceBuffer data;  // pipeline-precision input of one member
    };
    struct ClassState {
        ServerClass config;
        int priority = 0;  // stream priority of the class's slots (lower value = higher priority)
        std::deque<std::shared_ptr<Request>> queue;
        std::uint64_t inElems = 0, outElems = 0;
        bool f64 = true;
    };

    void loop();
    void launch(Slot& slot);
    void finish(Slot& slot);

    std::vector<ClassState> classes_;
    std::vector<std::unique_ptr<Slot>> slots_;
    std::map<std::uint64_t, std::shared_ptr<Request>> requests_;
    std::map<std::int64_t, State> states_;
    std::mutex mu_;
    std::condition_variable work_, done_;
    std::thread worker_;
    bool stop_ = false;
    bool held_ = false;
    int device_ = 0;
    std::uint64_t nextTicket_ = 1;
    std::int64_t nextState_ = 1;
    ServerStats stats_;
};

}  // namespace skb

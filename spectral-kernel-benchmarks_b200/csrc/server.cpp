#include "server.hpp"

#include <algorithm>

#include "util.hpp"

namespace skb {


Server::Server(const std::vector<ServerClass>& classes, std::uint64_t hbmBudget, int maxSlotsPerClass) {
    if (classes.empty()) throw Error(-1, "the server needs at least one size class");
    if (maxSlotsPerClass < 1) throw Error(-1, "at least one slot per size class");
    check_cuda(cudaGetDevice(&device_), "cudaGetDevice");
    stats_.budgetBytes = hbmBudget;
    for (const auto& c : classes) {
        if (c.maxBatch == 0) throw Error(-1, "maxBatch must be positive");
        ClassState cs;
        cs.config = c;
        const Workload w{c.n, c.n, c.nz, c.targets, 1.0, 1.0, true};
        const auto modes = retained_modes(w).size();
        cs.inElems = modes * (3 + 3 * c.targets) * w.nj();
        cs.outElems = modes * c.targets * w.nj();
        cs.f64 = c.mode == FluxMode::fp64_plain;
        classes_.push_back(std::move(cs));
    }
    // Stream priorities by size class: the class with the least work per
    // request gets the highest priority, so its kernels' CTAs are dispatched
    // ahead of the CTAs still waiting in a larger class's launches (running
    // CTAs are not preempted) and a small request is not held behind a
    // 512^2 batch.
    int leastPriority = 0, greatestPriority = 0;
    check_cuda(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority),
               "cudaDeviceGetStreamPriorityRange");
    {
        std::vector<int> order(classes_.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
        auto work = [&](int i) {
            const auto& c = classes_[i].config;
            return static_cast<double>(c.n) * c.n * c.nz * (3 + 4 * c.targets) * (c.mode == FluxMode::fp64_plain ? 2 : 1);
        };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) < work(b); });
        // Priorities count down from greatestPriority (numerically the lowest).
        int level = greatestPriority;
        for (size_t r = 0; r < order.size(); ++r) {
            if (r > 0 && work(order[r]) > work(order[r - 1]) && level < leastPriority) ++level;
            classes_[order[r]].priority = level;
        }
    }
    // Slots: one per class first (the minimum service), then more round-robin
    // while the footprint stays inside the budget.  A slot's footprint is the
    // sum of its own device allocations (the flux pipeline's persistent and
    // scratch buffers, the batch input / output and the FP64 staging), so other
    // allocations on the device cannot distort the accounting.
    auto makeSlot = [&](int cls) -> std::uint64_t {
        auto slot = std::make_unique<Slot>();
        slot->cls = cls;
        const auto& c = classes_[cls];
        FluxConfig fc;
        fc.n = c.config.n;
        fc.nz = c.config.nz;
        fc.targets = c.config.targets;
        fc.members = c.config.maxBatch;
        fc.mode = c.config.mode;
        slot->flux = std::make_unique<FluxPipeline>(fc);
        const size_t es = c.f64 ? 16 : 8;
        slot->in.allocate(es * c.inElems * fc.members);
        slot->out.allocate(es * c.outElems * fc.members);
        if (!c.f64) slot->stage.allocate(16 * std::max(c.inElems, c.outElems) * fc.members);
        check_cuda(cudaStreamCreateWithPriority(&slot->stream, cudaStreamNonBlocking, c.priority),
                   "cudaStreamCreateWithPriority");
        check_cuda(cudaEventCreateWithFlags(&slot->event, cudaEventDisableTiming), "cudaEventCreateWithFlags");
        const std::uint64_t bytes = slot->flux->persistentBytes + slot->flux->scratchBytes + slot->in.bytes() +
                                    slot->out.bytes() + slot->stage.bytes();
        stats_.slotBytes += bytes;
        slots_.push_back(std::move(slot));
        return bytes;
    };
    std::vector<std::uint64_t> perClass(classes_.size(), 0);
    for (int c = 0; c < static_cast<int>(classes_.size()); ++c) perClass[c] = makeSlot(c);
    if (stats_.slotBytes > hbmBudget)
        throw Error(-4, "admission refused: one slot per size class needs " + std::to_string(stats_.slotBytes) +
                            " device bytes, budget " + std::to_string(hbmBudget));
    for (int round = 1; round < maxSlotsPerClass; ++round) {
        for (int c = 0; c < static_cast<int>(classes_.size()); ++c) {
            if (stats_.slotBytes + perClass[c] > hbmBudget) continue;
            try {
                makeSlot(c);
            } catch (const Error& e) {
                if (e.code() != -4) throw;  // out of device memory: keep the slots made so far
            }
        }
    }
    stats_.slots = slots_.size();
    worker_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    work_.notify_all();
    if (worker_.joinable()) worker_.join();
    for (auto& s : slots_) {
        if (s->event) cudaEventDestroy(s->event);
        if (s->stream) cudaStreamDestroy(s->stream);
    }
}

std::uint64_t Server::inputElements(int cls) const {
    if (cls < 0 || cls >= static_cast<int>(classes_.size())) throw Error(-1, "unknown size class");
    return classes_[cls].inElems;
}

std::uint64_t Server::outputElements(int cls) const {
    if (cls < 0 || cls >= static_cast<int>(classes_.size())) throw Error(-1, "unknown size class");
    return classes_[cls].outElems;
}

std::uint64_t Server::submit(int cls, const double* input, double* output) {
    if (cls < 0 || cls >= static_cast<int>(classes_.size())) throw Error(-1, "unknown size class");
    if (input == nullptr || output == nullptr) throw Error(-1, "request buffers must be non-null");
    auto req = std::make_shared<Request>();
    req->cls = cls;
    req->input = input;
    req->output = output;
    req->submitted = Clock::now();
    std::uint64_t ticket;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (stop_) throw Error(-2, "the server is stopping");
        ticket = req->ticket = nextTicket_++;
        requests_[ticket] = req;
        classes_[cls].queue.push_back(req);
        ++stats_.submitted;
    }
    work_.notify_all();
    return ticket;
}

std::uint64_t Server::submitState(std::int64_t state, double* output) {
    if (output == nullptr) throw Error(-1, "request buffers must be non-null");
    auto req = std::make_shared<Request>();
    req->state = state;
    req->output = output;
    req->submitted = Clock::now();
    std::uint64_t ticket;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = states_.find(state);
        if (it == states_.end()) throw Error(-1, "unknown resident state");
        if (stop_) throw Error(-2, "the server is stopping");
        req->cls = it->second.cls;
        ticket = req->ticket = nextTicket_++;
        requests_[ticket] = req;
        classes_[req->cls].queue.push_back(req);
        ++stats_.submitted;
    }
    work_.notify_all();
    return ticket;
}

std::int64_t Server::loadState(int cls, const double* input) {
    if (cls < 0 || cls >= static_cast<int>(classes_.size())) throw Error(-1, "unknown size class");
    if (input == nullptr) throw Error(-1, "state input must be non-null");
    const auto& c = classes_[cls];
    const std::uint64_t bytes = c.inElems * (c.f64 ? 16 : 8);
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (stats_.slotBytes + stats_.stateBytes + bytes > stats_.budgetBytes)
            throw Error(-4, "admission refused: resident state of " + std::to_string(bytes) +
                                " bytes exceeds the remaining HBM budget");
        stats_.stateBytes += bytes;
    }
    State st;
    st.cls = cls;
    try {
        st.data.allocate(bytes);
        if (c.f64) {
            check_cuda(cudaMemcpy(st.data.get(), input, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
        } else {
            DeviceBuffer tmp(16 * c.inElems);
            check_cuda(cudaMemcpy(tmp.get(), input, 16 * c.inElems, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
            check_cuda(launch_convert_f64_to_f32(tmp.get<double>(), st.data.get<float>(),
                                                 static_cast<long long>(2 * c.inElems), nullptr),
                       "convert kernel");
            check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        }
    } catch (...) {
        std::lock_guard<std::mutex> lk(mu_);
        stats_.stateBytes -= bytes;
        throw;
    }
    std::lock_guard<std::mutex> lk(mu_);
    const auto id = nextState_++;
    states_.emplace(id, std::move(st));
    stats_.residentStates = states_.size();
    return id;
}

void Server::releaseState(std::int64_t state) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = states_.find(state);
    if (it == states_.end()) throw Error(-1, "unknown resident state");
    for (const auto& c : classes_)
        for (const auto& r : c.queue)
            if (r->state == state) throw Error(-3, "resident state still referenced by a queued request");
    for (const auto& s : slots_)
        for (const auto& r : s->batch)
            if (r->state == state) throw Error(-3, "resident state still referenced by a running batch");
    stats_.stateBytes -= it->second.data.bytes();
    states_.erase(it);
    stats_.residentStates = states_.size();
}

bool Server::wait(std::uint64_t ticket, double timeoutSeconds, double* latencyMs) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = requests_.find(ticket);
    if (it == requests_.end()) throw Error(-1, "unknown request ticket");
    auto req = it->second;
    const bool finished = done_.wait_for(lk, std::chrono::duration<double>(timeoutSeconds), [&] { return req->done; });
    if (!finished) return false;
    requests_.erase(ticket);
    if (latencyMs) *latencyMs = std::chrono::duration<double, std::milli>(req->finished - req->submitted).count();
    if (req->status != 0) throw Error(req->status, req->error);
    return true;
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lk(mu_);
    return stats_;
}

void Server::launch(Slot& slot) {
    auto& c = classes_[slot.cls];
    const auto take = std::min<std::uint64_t>(c.config.maxBatch, c.queue.size());
    for (std::uint64_t i = 0; i < take; ++i) {
        slot.batch.push_back(c.queue.front());
        c.queue.pop_front();
    }
    const size_t es = c.f64 ? 16 : 8;
    const auto inBytes = es * c.inElems, outBytes = es * c.outElems;
    try {
        for (std::uint64_t i = 0; i < take; ++i) {
            const auto& r = slot.batch[i];
            auto* dst = slot.in.get<unsigned char>() + i * inBytes;
            if (r->state >= 0) {
                const auto& st = states_.at(r->state);
                check_cuda(cudaMemcpyAsync(dst, st.data.get(), inBytes, cudaMemcpyDeviceToDevice, slot.stream),
                           "cudaMemcpyAsync D2D");
            } else if (c.f64) {
                check_cuda(cudaMemcpyAsync(dst, r->input, inBytes, cudaMemcpyHostToDevice, slot.stream),
                           "cudaMemcpyAsync H2D");
            } else {
                auto* stage = slot.stage.get<unsigned char>() + i * 16 * c.inElems;
                check_cuda(cudaMemcpyAsync(stage, r->input, 16 * c.inElems, cudaMemcpyHostToDevice, slot.stream),
                           "cudaMemcpyAsync H2D");
                check_cuda(launch_convert_f64_to_f32(reinterpret_cast<const double*>(stage),
                                                     reinterpret_cast<float*>(dst),
                                                     static_cast<long long>(2 * c.inElems), slot.stream),
                           "convert kernel");
            }
        }
        slot.flux->execute(slot.in.get(), slot.out.get(), slot.stream, take);
        if (!c.f64)
            check_cuda(launch_convert_f32_to_f64(slot.out.get<float>(), slot.stage.get<double>(),
                                                 static_cast<long long>(2 * c.outElems * take), slot.stream),
                       "convert kernel");
        const unsigned char* results = c.f64 ? slot.out.get<unsigned char>() : slot.stage.get<unsigned char>();
        for (std::uint64_t i = 0; i < take; ++i)
            check_cuda(cudaMemcpyAsync(slot.batch[i]->output, results + i * 16 * c.outElems, 16 * c.outElems,
                                       cudaMemcpyDeviceToHost, slot.stream),
                       "cudaMemcpyAsync D2H");
        check_cuda(cudaEventRecord(slot.event, slot.stream), "cudaEventRecord");
        (void)outBytes;
        slot.busy = true;
        ++stats_.batches;
    } catch (const Error& e) {
        for (auto& r : slot.batch) {
            r->status = e.code();
            r->error = e.what();
            r->finished = Clock::now();
            r->done = true;
            ++stats_.completed;
        }
        slot.batch.clear();
        done_.notify_all();
    }
}

void Server::finish(Slot& slot) {
    const auto now = Clock::now();
    int status = 0;
    std::string error;
    try {
        slot.flux->check_device_errors();
    } catch (const Error& e) {
        status = e.code();
        error = e.what();
    }
    for (auto& r : slot.batch) {
        r->finished = now;
        r->status = status;
        r->error = error;
        r->done = true;
        ++stats_.completed;
    }
    slot.batch.clear();
    slot.busy = false;
    done_.notify_all();
}

void Server::hold(bool held) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        held_ = held;
    }
    work_.notify_all();
}

void Server::loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    while (true) {
        bool progress = false;
        bool anyBusy = false;
        for (auto& s : slots_) {
            if (!s->busy) continue;
            const cudaError_t q = cudaEventQuery(s->event);
            if (q == cudaSuccess) {
                finish(*s);
                progress = true;
            } else if (q != cudaErrorNotReady) {
                for (auto& r : s->batch) {
                    r->status = -2;
                    r->error = std::string("flux batch failed: ") + cudaGetErrorString(q);
                    r->finished = Clock::now();
                    r->done = true;
                    ++stats_.completed;
                }
                s->batch.clear();
                s->busy = false;
                done_.notify_all();
                progress = true;
            } else {
                anyBusy = true;
            }
        }
        if (stop_) {
            if (anyBusy) {
                work_.wait_for(lk, std::chrono::microseconds(100));
                continue;
            }
            for (auto& c : classes_) {
                for (auto& r : c.queue) {
                    r->status = -2;
                    r->error = "the server stopped before the request ran";
                    r->finished = Clock::now();
                    r->done = true;
                }
                c.queue.clear();
            }
            done_.notify_all();
            break;
        }
        for (auto& s : slots_) {
            if (held_ || s->busy || classes_[s->cls].queue.empty()) continue;
            launch(*s);
            progress = true;
        }
        if (!progress) work_.wait_for(lk, std::chrono::microseconds(50));
    }
}

}  // namespace skb

// A continuous-batching server for encrypted vector x plaintext-matrix products
// (MatmulHelper's coefficient encoding, app/LinearHelper.cuh).
//
// MatmulServer serves a stream of single-row requests of different shapes: requests
// wait in a FIFO queue; whenever one of its `slots` streams is free it admits queued
// requests (oldest first) while their device footprint fits the memory budget, and
// runs them together as one wave (one set of launches over all admitted requests) on
// that stream. Waves on different streams overlap on the device. Each request's
// arithmetic depends only on its own data, so a result is the same whether the
// request ran alone or in a mix.
#pragma once

#include <chrono>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "linear.hpp"

namespace troyn {

class MatmulServer {
public:
    struct Options {
        std::size_t memory_budget = std::size_t(8) << 30;  // device bytes of admitted requests
        int slots = 3;                                     // waves in flight (one stream each)
        std::size_t max_wave_requests = 256;
        std::size_t output_staging = std::size_t(256) << 20;  // page-locked result bytes per slot
    };
    struct Stats {
        std::uint64_t submitted = 0, completed = 0, failed = 0, waves = 0;
        std::size_t peak_bytes = 0, max_wave = 0;
        double launch_host_s = 0, reap_host_s = 0;  // host time inside launch / reap
        double alloc_host_s = 0;                    // of launch: in the device allocator
        double device_s = 0;                        // sum of wave durations on the device
    };

    MatmulServer(const SEALContext &context, Options options);
    ~MatmulServer();
    MatmulServer(const MatmulServer &) = delete;
    MatmulServer &operator=(const MatmulServer &) = delete;

    // Seconds on the steady clock the server stamps completions with.
    static double now();

    // Queues one request: `inputs` are the encrypted input ciphertexts at the first
    // level, in order (plan.inputBlocks() ciphertexts of 2 x L x N words),
    // `weights` the row-major in x out matrix mod t. arrival is a now() stamp.
    // Returns the request id; throws std::invalid_argument on inconsistent sizes or a
    // request larger than the whole memory budget.
    std::uint64_t submit(std::size_t in, std::size_t out, const std::uint64_t *inputs, std::size_t input_words,
                         const std::uint64_t *weights, double arrival);
    // The same without copying at submission: `inputs` and `weights` are read when the
    // request is admitted, and `owner` (may be null) is held until they have been read;
    // the caller keeps the memory unchanged meanwhile. Page-locked (pinned) memory is
    // copied to the device directly; other memory goes through the slot's staging.
    // With `outputs` (plan.outputBlocks() x 2 x L x N words, page-locked for a direct
    // copy) the results are written there and result()/take() hand back no words.
    std::uint64_t submitBorrowed(std::size_t in, std::size_t out, const std::uint64_t *inputs,
                                 std::size_t input_words, const std::uint64_t *weights, double arrival,
                                 std::shared_ptr<void> owner, std::uint64_t *outputs = nullptr);
    // Non-blocking: collects finished waves, then launches new waves on free slots.
    // Returns the ids that finished during this call.
    std::vector<std::uint64_t> step();
    // Steps until every queued and running request has finished or `timeout` seconds
    // passed; returns false on timeout.
    bool drain(double timeout);
    bool idle() const { return queue_.empty() && running_.empty(); }
    std::size_t slotDegree() const { return n_; }
    std::size_t ciphertextWords() const { return 2 * (std::size_t)L_ * n_; }
    std::size_t queued() const { return queue_.size(); }
    // Output ciphertexts (plan.outputBlocks() x 2 x L x N words) of a finished request,
    // with its arrival and completion stamps; false if unknown or not finished.
    // `ok` is false for a request whose wave failed.
    bool result(std::uint64_t id, std::vector<std::uint64_t> &outputs, double &arrival, double &done, bool &ok);
    // result() that hands the outputs over without a copy and forgets the request.
    bool take(std::uint64_t id, std::vector<std::uint64_t> &outputs, double &arrival, double &done, bool &ok);
    void release(std::uint64_t id) { done_.erase(id); }
    const Stats &stats() const { return stats_; }
    // Makes the next launched wave report a failed library call (a host-side fault
    // injection for tests of the failure path; no device work is altered).
    void injectWaveFailure() { inject_ = true; }

private:
    struct Request {
        std::uint64_t id;
        std::size_t in, out;
        MatmulPlan plan;
        const std::uint64_t *in_ptr = nullptr, *w_ptr = nullptr;
        std::shared_ptr<void> owner;                  // keeps borrowed memory alive
        bool pinned = false;                          // both arrays page-locked: direct copies
        std::uint64_t *out_ptr = nullptr;             // caller's result buffer, if any
        bool out_pinned = false;
        double arrival;
        std::size_t bytes;
    };
    struct Wave;
    struct Staging;
    struct Done {
        std::vector<std::uint64_t> outputs;
        double arrival, done;
        bool ok;
    };
    std::size_t footprint(const MatmulPlan &p) const;
    bool launch(int slot);
    void reap(std::vector<std::uint64_t> &finished);

    const SEALContext &context_;
    Options opt_;
    int L_ = 0;
    std::size_t n_ = 0;
    std::uint64_t next_id_ = 1;
    std::size_t in_flight_bytes_ = 0;
    bool inject_ = false;
    std::deque<Request> queue_;
    std::vector<void *> streams_;
    std::vector<std::unique_ptr<Staging>> pins_;  // per slot: staged inputs, outputs
    std::map<int, std::unique_ptr<Wave>> running_;
    std::map<std::uint64_t, Done> done_;
    Stats stats_;
};

}  // namespace troyn

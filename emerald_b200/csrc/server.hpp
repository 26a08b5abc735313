// Request loop over one batch arena: scene-simulation requests are admitted
// while the arena (sized from a device-memory budget) has room, stay
// resident on the device until their sub-steps are done, and are stepped
// together with every other resident scene (continuous batching: a request
// that arrives while others run joins at the next admission point, and a
// finished one leaves and frees its room at once).
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

#include "../../include/emerald_sph.h"
#include "engine.hpp"

namespace emerald {

struct ServerRequest {
    int64_t id = 0;
    emerald_params params{};
    std::vector<float> solid_xy, solid_volumes, fluid_xy, fluid_v;
    uint32_t n_fluid = 0, n_solid = 0;
    int32_t substeps = 0;
    // filled by the loop
    int scene = -1;
    int32_t remaining = 0;
    std::chrono::steady_clock::time_point submitted, admitted, finished;
    bool done = false;
    int status = EMERALD_OK;
    std::vector<float> x, v;
    SceneState final_state{};
};

class Server {
public:
    explicit Server(emerald_server_config const& cfg);
    ~Server();
    Server(Server const&) = delete;
    Server& operator=(Server const&) = delete;

    // Queues a request (inputs are copied). Returns EMERALD_ENOSPC when the
    // scene can never fit the arena.
    int submit(std::unique_ptr<ServerRequest> r, int64_t& id);
    // Waits up to timeout_ms (negative: for ever) for the request's result,
    // copies it out and forgets the request. EMERALD_ETIMEOUT when not done.
    int wait(int64_t id, int32_t timeout_ms, float* x, float* v, emerald_step_stats* stats,
             emerald_request_timing* timing);
    void stats(emerald_server_stats& out);

private:
    void loop();
    void admit_locked(std::unique_lock<std::mutex>& lock);
    void retire(std::vector<ServerRequest*> const& finished);

    emerald_server_config cfg_;
    int device_ = 0;
    std::unique_ptr<Engine> engine_;
    std::thread worker_;
    std::mutex mu_;
    std::condition_variable work_cv_, done_cv_;
    bool stop_ = false;
    int64_t next_id_ = 1;
    std::deque<std::unique_ptr<ServerRequest>> queue_;
    std::vector<std::unique_ptr<ServerRequest>> running_;
    std::map<int64_t, std::unique_ptr<ServerRequest>> finished_;
    int loop_status_ = EMERALD_OK;

    // statistics (guarded by mu_)
    int64_t submitted_ = 0, completed_ = 0, rejected_ = 0;
    int64_t batch_substeps_ = 0, scene_substeps_ = 0;
    double particle_substeps_ = 0.0;
    double busy_seconds_ = 0.0;
    int32_t resident_peak_ = 0;
    std::vector<float> step_ms_, request_ms_, queue_ms_;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};

}  // namespace emerald

// Request loop over batch arenas: scene-simulation requests are admitted
// while an arena (sized from a device-memory budget) has room, stay resident
// on the device until their sub-steps are done, and are stepped together
// with every other scene of their arena (continuous batching: a request that
// arrives while others run joins at the next admission point, and a finished
// one leaves and frees its room at once).
//
// The budget is split over a few lanes, each an arena with its own stream
// and worker thread. The scenes of one arena advance in lock step, so a
// sub-step lasts as long as its slowest scene's solver loop; while one lane
// runs the last iterations of a few unconverged scenes (small launches),
// the other lanes' sub-steps fill the GPU.
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
    int lane = -1;
    int scene = -1;
    int32_t remaining = 0;
    std::chrono::steady_clock::time_point submitted, admitted, finished;
    int status = EMERALD_OK;
    bool cancel = false;  // retire at the lane's next admission point
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
    // scene can never fit an arena.
    int submit(std::unique_ptr<ServerRequest> r, int64_t& id);
    // Waits up to timeout_ms (negative: for ever) for the request's result,
    // copies it out and forgets the request. EMERALD_ETIMEOUT when not done.
    int wait(int64_t id, int32_t timeout_ms, float* x, float* v, emerald_step_stats* stats,
             emerald_request_timing* timing);
    void stats(emerald_server_stats& out);
    // Cancels a queued, resident or finished request (emerald_server_cancel).
    int cancel(int64_t id);

private:
    struct Lane {
        int index = 0;
        std::unique_ptr<Engine> engine;
        cudaStream_t stream = nullptr;
        // marks[s] and marks[s + 1] bracket sub-step s of a launch round
        std::vector<cudaEvent_t> marks;
        std::thread worker;
        std::vector<std::unique_ptr<ServerRequest>> running;
        // guarded by mu_
        Engine::Room room{};
        double resident_particles = 0.0;
        double resident_work = 0.0;  // sum of fluid particles x sub-steps left
    };

    void loop(Lane& lane);
    // Lane that request r should join now: the one with room and the least
    // resident work.
    int preferred_lane(ServerRequest const& r) const;
    void admit_locked(Lane& lane);
    // Retires the lane's resident requests marked for cancellation.
    void retire_cancelled_locked(Lane& lane);
    void resident_changed_locked(int delta);

    emerald_server_config cfg_;
    int device_ = 0;
    std::vector<std::unique_ptr<Lane>> lanes_;
    mutable std::mutex mu_;
    std::condition_variable work_cv_, done_cv_;
    bool stop_ = false;
    uint64_t version_ = 0;  // bumped on every submit, admission and retirement
    int64_t next_id_ = 1;
    std::deque<std::unique_ptr<ServerRequest>> queue_;
    std::map<int64_t, std::unique_ptr<ServerRequest>> finished_;
    int loop_status_ = EMERALD_OK;

    // statistics (guarded by mu_)
    int64_t submitted_ = 0, completed_ = 0, rejected_ = 0, cancelled_ = 0;
    int64_t batch_substeps_ = 0, scene_substeps_ = 0;
    double particle_substeps_ = 0.0;
    double busy_seconds_ = 0.0;
    int resident_ = 0;
    std::chrono::steady_clock::time_point busy_since_;
    int32_t resident_peak_ = 0;
    std::vector<float> step_ms_, request_ms_, queue_ms_;
};

}  // namespace emerald

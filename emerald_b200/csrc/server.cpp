// Request loop over batch arenas (see server.hpp).
#include "server.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace emerald {

namespace {

// Fluid and boundary capacities that fit `budget` device bytes, with equal
// fluid and boundary capacity (a dam-break block of n particles has about
// 18 sqrt(n) boundary particles, below n for n >= 324; a boundary particle
// costs a twentieth of a fluid one).
void capacities(size_t budget, int scenes, uint32_t& fluid, uint32_t& solid) {
    uint64_t lo = kTile, hi = uint64_t(1) << 30;
    if (Engine::footprint(uint32_t(lo), uint32_t(lo), scenes) > budget) {
        throw std::runtime_error("device memory budget below the smallest arena");
    }
    while (hi - lo > kTile) {
        uint64_t const mid = (lo + hi) / 2 / kTile * kTile;
        if (Engine::footprint(uint32_t(mid), uint32_t(mid), scenes) <= budget) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    fluid = uint32_t(lo);
    solid = uint32_t(lo);
}

float percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.0f;
    std::sort(v.begin(), v.end());
    double const pos = q * double(v.size() - 1);
    size_t const k = size_t(pos);
    double const f = pos - double(k);
    double const hi = v[std::min(k + 1, v.size() - 1)];
    return float(double(v[k]) * (1.0 - f) + hi * f);
}

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

Server::Server(emerald_server_config const& cfg) : cfg_(cfg) {
    if (cfg_.max_scenes < 1) cfg_.max_scenes = 1;
    if (cfg_.max_substeps_per_launch < 1) cfg_.max_substeps_per_launch = 8;
    if (cfg_.lanes < 1) cfg_.lanes = 4;
    if (cfg_.order != 1) cfg_.order = 0;
    if (cudaGetDevice(&device_) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("no current CUDA device");
    }
    int const per_lane_scenes = (cfg_.max_scenes + cfg_.lanes - 1) / cfg_.lanes;
    size_t const per_lane_budget = cfg_.hbm_budget_bytes / size_t(cfg_.lanes);
    for (int k = 0; k < cfg_.lanes; ++k) {
        std::unique_ptr<Lane> lane(new Lane);
        lane->index = k;
        uint32_t fluid = 0, solid = 0;
        capacities(per_lane_budget, per_lane_scenes, fluid, solid);
        lane->engine.reset(new Engine(fluid, solid, per_lane_scenes));
        if (cudaStreamCreateWithFlags(&lane->stream, cudaStreamNonBlocking) != cudaSuccess) {
            throw std::runtime_error("stream creation failed");
        }
        lane->marks.resize(size_t(cfg_.max_substeps_per_launch) + 1);
        for (auto& e : lane->marks) {
            if (cudaEventCreate(&e) != cudaSuccess) throw std::runtime_error("event creation failed");
        }
        lane->engine->set_stream(lane->stream);
        lane->room = lane->engine->room();
        lanes_.push_back(std::move(lane));
    }
    for (auto& lane : lanes_) {
        Lane* l = lane.get();
        l->worker = std::thread([this, l] { loop(*l); });
    }
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_ = true;
    }
    work_cv_.notify_all();
    for (auto& lane : lanes_) {
        if (lane->worker.joinable()) lane->worker.join();
    }
    for (auto& lane : lanes_) {
        lane->engine.reset();
        if (lane->stream) cudaStreamDestroy(lane->stream);
        for (auto e : lane->marks) {
            if (e) cudaEventDestroy(e);
        }
    }
}

int Server::submit(std::unique_ptr<ServerRequest> r, int64_t& id) {
    std::lock_guard<std::mutex> lock(mu_);
    if (loop_status_ != EMERALD_OK) return loop_status_;
    bool fits_empty = false;
    for (auto const& lane : lanes_) {
        fits_empty = fits_empty ||
                     (r->n_fluid <= lane->engine->fluid_capacity() &&
                      r->n_solid <= lane->engine->solid_capacity());
    }
    if (!fits_empty) {
        ++rejected_;
        return EMERALD_ENOSPC;
    }
    r->id = next_id_++;
    r->remaining = r->substeps;
    r->submitted = std::chrono::steady_clock::now();
    id = r->id;
    if (cfg_.order == 1) {
        // largest work first; equal work keeps arrival order
        double const w = double(r->n_fluid) * double(r->substeps);
        auto pos = queue_.begin();
        while (pos != queue_.end() &&
               double((*pos)->n_fluid) * double((*pos)->substeps) >= w) {
            ++pos;
        }
        queue_.insert(pos, std::move(r));
    } else {
        queue_.push_back(std::move(r));
    }
    ++submitted_;
    ++version_;
    work_cv_.notify_all();
    return EMERALD_OK;
}

int Server::preferred_lane(ServerRequest const& r) const {
    int best = -1;
    for (auto const& lane : lanes_) {
        if (!lane->room.fits(r.n_fluid, r.n_solid)) continue;
        if (best < 0 || lane->resident_work < lanes_[size_t(best)]->resident_work) {
            best = lane->index;
        }
    }
    return best;
}

void Server::resident_changed_locked(int delta) {
    auto const now = std::chrono::steady_clock::now();
    if (resident_ == 0 && delta > 0) busy_since_ = now;
    resident_ += delta;
    if (resident_ == 0 && delta < 0) busy_seconds_ += ms_between(busy_since_, now) / 1000.0;
    resident_peak_ = std::max<int32_t>(resident_peak_, resident_);
}

// First fit in queue order: every queued request for which this lane is
// the lane with room and the least resident work joins this lane's batch; a
// large request that fits nowhere yet keeps its place while smaller ones
// behind it start.
void Server::admit_locked(Lane& lane) {
    for (auto it = queue_.begin(); it != queue_.end();) {
        ServerRequest& r = **it;
        if (preferred_lane(r) != lane.index) {
            ++it;
            continue;
        }
        SceneSpec spec;
        spec.params = r.params;
        spec.method = cfg_.method;
        spec.mode = kFrame;
        spec.solid_xy = r.solid_xy.data();
        spec.solid_volumes = r.solid_volumes.empty() ? nullptr : r.solid_volumes.data();
        spec.n_solid = r.n_solid;
        spec.fluid_xy = r.fluid_xy.data();
        spec.fluid_v = r.fluid_v.empty() ? nullptr : r.fluid_v.data();
        spec.n_fluid = r.n_fluid;
        int const scene = lane.engine->add_scene(spec);
        lane.room = lane.engine->room();
        if (scene < 0) {
            ++it;
            continue;
        }
        lane.engine->set_active(scene, true);
        r.lane = lane.index;
        r.scene = scene;
        r.admitted = std::chrono::steady_clock::now();
        queue_ms_.push_back(float(ms_between(r.submitted, r.admitted)));
        // inputs are on the device now
        std::vector<float>().swap(r.solid_xy);
        std::vector<float>().swap(r.solid_volumes);
        std::vector<float>().swap(r.fluid_xy);
        std::vector<float>().swap(r.fluid_v);
        lane.resident_particles += double(r.n_fluid);
        lane.resident_work += double(r.n_fluid) * double(r.remaining);
        lane.running.push_back(std::move(*it));
        it = queue_.erase(it);
        resident_changed_locked(+1);
        ++version_;
    }
}

void Server::retire_cancelled_locked(Lane& lane) {
    auto const now = std::chrono::steady_clock::now();
    for (auto it = lane.running.begin(); it != lane.running.end();) {
        ServerRequest& r = **it;
        if (!r.cancel) {
            ++it;
            continue;
        }
        lane.engine->remove_scene(r.scene);
        lane.room = lane.engine->room();
        lane.resident_particles -= double(r.n_fluid);
        lane.resident_work = std::max(0.0, lane.resident_work -
                                               double(r.n_fluid) * double(std::max(r.remaining, 0)));
        r.status = EMERALD_ECANCELED;
        r.finished = now;
        resident_changed_locked(-1);
        finished_[r.id] = std::move(*it);
        it = lane.running.erase(it);
        ++version_;
        done_cv_.notify_all();
    }
}

int Server::cancel(int64_t id) {
    std::lock_guard<std::mutex> lock(mu_);
    for (auto it = queue_.begin(); it != queue_.end(); ++it) {
        if ((*it)->id != id) continue;
        (*it)->status = EMERALD_ECANCELED;
        (*it)->finished = std::chrono::steady_clock::now();
        finished_[id] = std::move(*it);
        queue_.erase(it);
        ++cancelled_;
        ++version_;
        done_cv_.notify_all();
        return EMERALD_OK;
    }
    for (auto const& lane : lanes_) {
        for (auto const& r : lane->running) {
            if (r->id != id) continue;
            if (!r->cancel) ++cancelled_;
            r->cancel = true;
            ++version_;
            work_cv_.notify_all();
            return EMERALD_OK;
        }
    }
    auto it = finished_.find(id);
    if (it == finished_.end()) return EMERALD_ENOTFOUND;
    if (it->second->status != EMERALD_ECANCELED) {
        it->second->status = EMERALD_ECANCELED;
        std::vector<float>().swap(it->second->x);
        std::vector<float>().swap(it->second->v);
        ++cancelled_;
    }
    return EMERALD_OK;
}

void Server::loop(Lane& lane) {
    cudaSetDevice(device_);
    Engine& engine = *lane.engine;
    std::unique_lock<std::mutex> lock(mu_);
    while (true) {
        uint64_t const seen = version_;
        if (!stop_ && loop_status_ == EMERALD_OK) {
            try {
                retire_cancelled_locked(lane);
                admit_locked(lane);
            } catch (std::exception const&) {
                loop_status_ = EMERALD_ECUDA;
            }
        }
        if (version_ != seen) work_cv_.notify_all();
        if (stop_ || loop_status_ != EMERALD_OK) {
            // drop what is resident: results of a stopped server are not read
            for (auto& r : lane.running) {
                try {
                    engine.remove_scene(r->scene);
                } catch (std::exception const&) {
                }
                resident_changed_locked(-1);
            }
            lane.running.clear();
            lane.resident_particles = 0.0;
            lane.resident_work = 0.0;
            done_cv_.notify_all();
            break;
        }
        if (lane.running.empty()) {
            uint64_t const now_seen = version_;
            work_cv_.wait(lock, [&] { return stop_ || version_ != now_seen; });
            continue;
        }
        int32_t k = cfg_.max_substeps_per_launch;
        double particles = 0.0;
        for (auto const& r : lane.running) {
            k = std::min(k, r->remaining);
            particles += double(r->n_fluid);
        }
        size_t const resident = lane.running.size();
        lock.unlock();
        std::vector<float> step_ms(size_t(std::max(k, 0)));
        int status = EMERALD_OK;
        try {
            // the round's sub-steps back to back, one host wait at the end
            cudaEventRecord(lane.marks[0], lane.stream);
            for (int32_t s = 0; s < k; ++s) {
                engine.substep(cfg_.method);
                cudaEventRecord(lane.marks[size_t(s) + 1], lane.stream);
            }
            cudaEventSynchronize(lane.marks[size_t(k)]);
            for (int32_t s = 0; s < k; ++s) {
                cudaEventElapsedTime(&step_ms[size_t(s)], lane.marks[size_t(s)],
                                     lane.marks[size_t(s) + 1]);
            }
            engine.check("server sub-step");
        } catch (std::exception const&) {
            status = EMERALD_ECUDA;
        }
        std::vector<ServerRequest*> fin;
        lock.lock();
        for (auto& r : lane.running) {
            r->remaining -= k;
            if (r->remaining <= 0 && !r->cancel) fin.push_back(r.get());
        }
        lock.unlock();
        if (status == EMERALD_OK) {
            try {
                for (ServerRequest* r : fin) {
                    r->x.resize(2ull * r->n_fluid);
                    r->v.resize(2ull * r->n_fluid);
                    engine.get_state(r->scene, r->x.data(), r->v.data());
                    r->final_state = engine.scene_state(r->scene);
                    engine.remove_scene(r->scene);
                    r->scene = -1;
                }
            } catch (std::exception const&) {
                status = EMERALD_ECUDA;
            }
        }
        lock.lock();
        step_ms_.insert(step_ms_.end(), step_ms.begin(), step_ms.end());
        batch_substeps_ += k;
        scene_substeps_ += int64_t(k) * int64_t(resident);
        particle_substeps_ += double(k) * particles;
        lane.resident_work = std::max(0.0, lane.resident_work - double(k) * particles);
        lane.room = engine.room();
        auto const now = std::chrono::steady_clock::now();
        for (auto it = lane.running.begin(); it != lane.running.end();) {
            ServerRequest& r = **it;
            if (status == EMERALD_OK && r.remaining > 0) {
                ++it;
                continue;
            }
            // a request cancelled during its last round keeps no result
            r.status = (status == EMERALD_OK && r.cancel) ? EMERALD_ECANCELED : status;
            r.finished = now;
            if (r.status == EMERALD_OK) {
                request_ms_.push_back(float(ms_between(r.submitted, r.finished)));
                ++completed_;
            } else if (r.cancel && r.scene >= 0) {
                engine.remove_scene(r.scene);
                r.scene = -1;
                lane.room = engine.room();
            }
            lane.resident_particles -= double(r.n_fluid);
            resident_changed_locked(-1);
            finished_[r.id] = std::move(*it);
            it = lane.running.erase(it);
        }
        if (status != EMERALD_OK) loop_status_ = status;
        if (!fin.empty() || status != EMERALD_OK) {
            ++version_;
            work_cv_.notify_all();
            done_cv_.notify_all();
        }
    }
}

int Server::wait(int64_t id, int32_t timeout_ms, float* x, float* v, emerald_step_stats* stats,
                 emerald_request_timing* timing) {
    std::unique_lock<std::mutex> lock(mu_);
    auto known = [&] {
        if (finished_.count(id)) return true;
        for (auto const& r : queue_) {
            if (r->id == id) return true;
        }
        for (auto const& lane : lanes_) {
            for (auto const& r : lane->running) {
                if (r->id == id) return true;
            }
        }
        return false;
    };
    if (!known()) return EMERALD_ENOTFOUND;
    auto ready = [&] { return finished_.count(id) != 0 || loop_status_ != EMERALD_OK || stop_; };
    if (timeout_ms < 0) {
        done_cv_.wait(lock, ready);
    } else if (!done_cv_.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready)) {
        return EMERALD_ETIMEOUT;
    }
    auto it = finished_.find(id);
    if (it == finished_.end()) return loop_status_ != EMERALD_OK ? loop_status_ : EMERALD_ETIMEOUT;
    std::unique_ptr<ServerRequest> r = std::move(it->second);
    finished_.erase(it);
    lock.unlock();
    if (r->status != EMERALD_OK) return r->status;
    if (x) std::copy(r->x.begin(), r->x.end(), x);
    if (v) std::copy(r->v.begin(), r->v.end(), v);
    if (stats) {
        SceneState const& s = r->final_state;
        stats->sub_steps = r->substeps;
        stats->pressure_iterations = s.stat_iters;
        stats->error_average = s.stat_avg;
        stats->error_max = s.stat_max;
        stats->divergence_iterations = s.stat_div_iters;
        stats->divergence_error_average = s.stat_div_avg;
        stats->divergence_error_max = s.stat_div_max;
        stats->dt = s.dt;
        stats->time_seconds = double(s.frame_time + s.elapsed) / 705600000.0;
        stats->error_flags = s.error;
        stats->error_average_exact = s.stat_avg_exact;
        stats->divergence_error_average_exact = s.stat_div_avg_exact;
    }
    if (timing) {
        timing->queue_ms = ms_between(r->submitted, r->admitted);
        timing->run_ms = ms_between(r->admitted, r->finished);
        timing->total_ms = ms_between(r->submitted, r->finished);
    }
    return EMERALD_OK;
}

void Server::stats(emerald_server_stats& out) {
    std::lock_guard<std::mutex> lock(mu_);
    out = emerald_server_stats{};
    out.submitted = submitted_;
    out.completed = completed_;
    out.rejected = rejected_;
    out.queued = int64_t(queue_.size());
    out.resident = int64_t(resident_);
    out.batch_substeps = batch_substeps_;
    out.scene_substeps = scene_substeps_;
    out.particle_substeps = particle_substeps_;
    out.busy_seconds = busy_seconds_;
    out.step_ms_p50 = percentile(step_ms_, 0.50);
    out.step_ms_p99 = percentile(step_ms_, 0.99);
    out.request_ms_p50 = percentile(request_ms_, 0.50);
    out.request_ms_p99 = percentile(request_ms_, 0.99);
    out.queue_ms_p50 = percentile(queue_ms_, 0.50);
    out.queue_ms_p99 = percentile(queue_ms_, 0.99);
    for (auto const& lane : lanes_) {
        out.fluid_capacity = std::max<size_t>(out.fluid_capacity, lane->engine->fluid_capacity());
        out.solid_capacity = std::max<size_t>(out.solid_capacity, lane->engine->solid_capacity());
        out.device_bytes += lane->engine->device_bytes();
    }
    out.resident_peak = resident_peak_;
    out.status = loop_status_;
    out.cancelled = cancelled_;
}

}  // namespace emerald

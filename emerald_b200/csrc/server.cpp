// Request loop over one batch arena (see server.hpp).
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
    uint32_t fluid = 0, solid = 0;
    capacities(cfg_.hbm_budget_bytes, cfg_.max_scenes, fluid, solid);
    if (cudaGetDevice(&device_) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("no current CUDA device");
    }
    engine_.reset(new Engine(fluid, solid, cfg_.max_scenes));
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        throw std::runtime_error("stream creation failed");
    }
    engine_->set_stream(st);
    if (cudaEventCreate(&ev0_) != cudaSuccess || cudaEventCreate(&ev1_) != cudaSuccess) {
        throw std::runtime_error("event creation failed");
    }
    worker_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_ = true;
    }
    work_cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    cudaStream_t const st = engine_ ? engine_->stream() : nullptr;
    engine_.reset();
    if (st) cudaStreamDestroy(st);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
}

int Server::submit(std::unique_ptr<ServerRequest> r, int64_t& id) {
    std::lock_guard<std::mutex> lock(mu_);
    if (loop_status_ != EMERALD_OK) return loop_status_;
    if (r->n_fluid > engine_->fluid_capacity() || r->n_solid > engine_->solid_capacity()) {
        ++rejected_;
        return EMERALD_ENOSPC;
    }
    r->id = next_id_++;
    r->remaining = r->substeps;
    r->submitted = std::chrono::steady_clock::now();
    id = r->id;
    queue_.push_back(std::move(r));
    ++submitted_;
    work_cv_.notify_all();
    return EMERALD_OK;
}

// First fit in arrival order: every queued request that the arena has room
// for now joins the batch; a large request that does not fit yet keeps its
// place while smaller ones behind it start.
void Server::admit_locked(std::unique_lock<std::mutex>& lock) {
    (void)lock;
    for (auto it = queue_.begin(); it != queue_.end();) {
        ServerRequest& r = **it;
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
        int const scene = engine_->add_scene(spec);
        if (scene < 0) {
            ++it;
            continue;
        }
        engine_->set_active(scene, true);
        r.scene = scene;
        r.admitted = std::chrono::steady_clock::now();
        queue_ms_.push_back(float(ms_between(r.submitted, r.admitted)));
        // inputs are on the device now
        std::vector<float>().swap(r.solid_xy);
        std::vector<float>().swap(r.solid_volumes);
        std::vector<float>().swap(r.fluid_xy);
        std::vector<float>().swap(r.fluid_v);
        running_.push_back(std::move(*it));
        it = queue_.erase(it);
    }
    resident_peak_ = std::max<int32_t>(resident_peak_, int32_t(running_.size()));
}

void Server::retire(std::vector<ServerRequest*> const& finished) {
    for (ServerRequest* r : finished) {
        r->x.resize(2ull * r->n_fluid);
        r->v.resize(2ull * r->n_fluid);
        engine_->get_state(r->scene, r->x.data(), r->v.data());
        r->final_state = engine_->scene_state(r->scene);
        engine_->remove_scene(r->scene);
    }
}

void Server::loop() {
    cudaSetDevice(device_);
    auto busy_since = std::chrono::steady_clock::now();
    bool busy = false;
    std::unique_lock<std::mutex> lock(mu_);
    while (true) {
        try {
            admit_locked(lock);
        } catch (std::exception const&) {
            loop_status_ = EMERALD_ECUDA;
        }
        if (running_.empty()) {
            if (busy) {
                busy_seconds_ += ms_between(busy_since, std::chrono::steady_clock::now()) / 1000.0;
                busy = false;
            }
            if (stop_ || loop_status_ != EMERALD_OK) break;
            work_cv_.wait(lock, [this] { return stop_ || !queue_.empty(); });
            continue;
        }
        if (!busy) {
            busy = true;
            busy_since = std::chrono::steady_clock::now();
        }
        if (stop_ || loop_status_ != EMERALD_OK) {
            // drop what is resident: results of a stopped server are not read
            for (auto& r : running_) engine_->remove_scene(r->scene);
            running_.clear();
            continue;
        }
        int32_t k = cfg_.max_substeps_per_launch;
        double particles = 0.0;
        for (auto const& r : running_) {
            k = std::min(k, r->remaining);
            particles += double(r->n_fluid);
        }
        size_t const resident = running_.size();
        lock.unlock();
        std::vector<float> step_ms(size_t(std::max(k, 0)));
        int status = EMERALD_OK;
        try {
            for (int32_t s = 0; s < k; ++s) {
                cudaEventRecord(ev0_, engine_->stream());
                engine_->substep(cfg_.method);
                cudaEventRecord(ev1_, engine_->stream());
                cudaEventSynchronize(ev1_);
                cudaEventElapsedTime(&step_ms[size_t(s)], ev0_, ev1_);
            }
            engine_->check("server sub-step");
        } catch (std::exception const&) {
            status = EMERALD_ECUDA;
        }
        lock.lock();
        if (status != EMERALD_OK) {
            loop_status_ = status;
            for (auto& r : running_) {
                r->done = true;
                r->status = status;
                r->finished = std::chrono::steady_clock::now();
                finished_[r->id] = std::move(r);
            }
            running_.clear();
            done_cv_.notify_all();
            continue;
        }
        step_ms_.insert(step_ms_.end(), step_ms.begin(), step_ms.end());
        batch_substeps_ += k;
        scene_substeps_ += int64_t(k) * int64_t(resident);
        particle_substeps_ += double(k) * particles;
        std::vector<ServerRequest*> fin;
        for (auto& r : running_) {
            r->remaining -= k;
            if (r->remaining <= 0) fin.push_back(r.get());
        }
        if (!fin.empty()) {
            lock.unlock();
            try {
                retire(fin);
            } catch (std::exception const&) {
                status = EMERALD_ECUDA;
            }
            lock.lock();
            auto const now = std::chrono::steady_clock::now();
            for (auto it = running_.begin(); it != running_.end();) {
                if ((*it)->remaining <= 0) {
                    ServerRequest& r = **it;
                    r.done = true;
                    r.status = status;
                    r.finished = now;
                    request_ms_.push_back(float(ms_between(r.submitted, r.finished)));
                    ++completed_;
                    finished_[r.id] = std::move(*it);
                    it = running_.erase(it);
                } else {
                    ++it;
                }
            }
            if (status != EMERALD_OK) loop_status_ = status;
            done_cv_.notify_all();
        }
    }
    lock.unlock();
    done_cv_.notify_all();
}

int Server::wait(int64_t id, int32_t timeout_ms, float* x, float* v, emerald_step_stats* stats,
                 emerald_request_timing* timing) {
    std::unique_lock<std::mutex> lock(mu_);
    auto ready = [&] { return finished_.count(id) != 0 || loop_status_ != EMERALD_OK; };
    bool known = finished_.count(id) != 0;
    if (!known) {
        for (auto const& r : queue_) known = known || r->id == id;
        for (auto const& r : running_) known = known || r->id == id;
    }
    if (!known) return EMERALD_ENOTFOUND;
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
    out.resident = int64_t(running_.size());
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
    out.fluid_capacity = engine_->fluid_capacity();
    out.solid_capacity = engine_->solid_capacity();
    out.device_bytes = engine_->device_bytes();
    out.resident_peak = resident_peak_;
    out.status = loop_status_;
}

}  // namespace emerald

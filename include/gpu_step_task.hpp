// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Hedgehog graph nodes of the GPU step, source-compatible with the
// reference's include/gpu_step_task.hpp:39-451 (same class names,
// constructors, members used by drivers, CSV/binary output formats), running
// on liblpbf_b200:
//
//   GpuStepTask        AbstractCUDATask<1, Tick, Tick, MetricsMsg, SnapshotMsg>
//                      advances a batch of steps per activation and
//                      recirculates the next batch's Tick to itself.
//                        mode 2, fused  -> lpbf_b200_advance: up to `depth`
//                                          steps per launch, step + reduce +
//                                          finalize fused (one launch per
//                                          group instead of 2 per step)
//                        mode 2, !fused -> per step: lpbf_launch_step,
//                                          lpbf_launch_reduce,
//                                          lpbf_launch_reduce_finalize
//                        mode 0 / 1     -> per step with host finalize and a
//                                          strided hot-column copy (mode 1:
//                                          only on cruise steps)
//                      A launch ends on every step whose field must exist on
//                      the device (hot column on cruise steps, snapshots).
//   MetricsTask        melt widths W and W_sub, running maxima, metrics.csv.
//   SnapshotWriterTask T_step_%06d.bin (raw row-major f64 field).
//
// All modes give byte-identical metrics and fields.
// ---------------------------------------------------------------------------
#pragma once

#include <hedgehog.h>   // real Hedgehog, or hedgehog_lpbf_b200/compat (HH_USE_CUDA)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "params.hpp"
#include "lpbf_step_const.hpp"
#include "lpbf_kernels.hpp"
#include "lpbf_b200.h"
#include "gpu_messages.hpp"

namespace lpbf {

// Running maxima filled in by MetricsTask (single-threaded).
struct RunAccum {
    double peak_T = 0.0;
    double peak_W = 0.0;
    double steady_W_sub = 0.0;
    std::int64_t steps_seen = 0;
};

// Cruise window of the single-track metrics: before the first wrap, laser
// between 45 % and 85 % of the domain length.
inline bool cruise_step(double x_laser_csv, bool wrapped, double Lx) {
    return !wrapped && x_laser_csv >= 0.45 * Lx && x_laser_csv <= 0.85 * Lx;
}

class GpuStepTask
    : public hh::AbstractCUDATask<1, Tick, Tick, MetricsMsg, SnapshotMsg> {
public:
    GpuStepTask(Domain dom, StepConst k, int phys_i, double Tm, int n_steps,
                std::vector<Tick> plan, double Tamb, bool write_outputs, int batch,
                int mode = 2, bool fused = false, bool pinned = false)
        : hh::AbstractCUDATask<1, Tick, Tick, MetricsMsg, SnapshotMsg>("GPU-Step", 1),
          dom_(dom), k_(k), phys_(phys_i), Tm_(Tm), n_steps_(n_steps),
          plan_(std::move(plan)), Tamb_(Tamb), write_outputs_(write_outputs),
          batch_(std::max(1, batch)), mode_(mode), fused_(fused), pinned_(pinned) {
        nx_ = dom_.nx;
        ny_ = dom_.ny;
        N_ = static_cast<std::size_t>(nx_) * ny_;
        nblk_reduce_ = static_cast<int>(std::min<long long>(256, ((long long)N_ + 255) / 256));
        nblk_fused_ = ((nx_ + 15) / 16) * ((ny_ + 15) / 16);
    }

    // Time steps per launch for the fused path (0 = library default).
    void depth(int d) { depth_ = d; }

    void initializeCuda() override {
        checkCudaErrors(cudaMalloc(&d_a_, N_ * sizeof(double)));
        checkCudaErrors(cudaMalloc(&d_b_, N_ * sizeof(double)));
        checkCudaErrors(cudaMalloc(&d_parts_, std::max(nblk_reduce_, nblk_fused_) * sizeof(Partial)));
        checkCudaErrors(cudaMalloc(&d_ring_, batch_ * sizeof(Partial)));
        checkCudaErrors(cudaMalloc(&d_cols_, (std::size_t)batch_ * ny_ * sizeof(double)));
        work_bytes_ = lpbf_b200_workspace_bytes();
        checkCudaErrors(cudaMalloc(&d_work_, work_bytes_));
        if (lpbf_b200_workspace_init(d_work_, work_bytes_, this->stream()) != LPBF_OK)
            throw std::runtime_error("lpbf_b200_workspace_init failed");
        if (pinned_) {
            checkCudaErrors(cudaHostAlloc(reinterpret_cast<void**>(&h_ring_),
                                          batch_ * sizeof(Partial), cudaHostAllocDefault));
            checkCudaErrors(cudaHostAlloc(reinterpret_cast<void**>(&h_cols_),
                                          (std::size_t)batch_ * ny_ * sizeof(double),
                                          cudaHostAllocDefault));
        } else {
            ring_store_.resize(batch_);
            cols_store_.resize((std::size_t)batch_ * ny_);
            h_ring_ = ring_store_.data();
            h_cols_ = cols_store_.data();
        }
        parts_store_.resize(nblk_reduce_);
        const std::vector<double> init(N_, Tamb_);
        checkCudaErrors(cudaMemcpy(d_a_, init.data(), N_ * sizeof(double),
                                   cudaMemcpyHostToDevice));
        cur_ = d_a_;
        nxt_ = d_b_;
    }

    void shutdownCuda() override {
        cudaFree(d_a_); cudaFree(d_b_); cudaFree(d_parts_);
        cudaFree(d_ring_); cudaFree(d_cols_); cudaFree(d_work_);
        if (pinned_) { cudaFreeHost(h_ring_); cudaFreeHost(h_cols_); }
    }

    void execute(std::shared_ptr<Tick> tick) override {
        if (mode_ == 0 || mode_ == 1) { per_step(*tick, mode_ == 1); return; }
        const int first = tick->step;
        const int last = std::min(first + batch_, n_steps_);     // exclusive
        struct Pending { int step; std::shared_ptr<std::vector<double>> field; };
        std::vector<Pending> snaps;

        int s = first;
        while (s < last) {
            // The group [s, e) ends at the first step whose field is needed.
            const int cap = fused_ ? group_cap() : 1;
            int e = s + 1;
            while (e < last && e - s < cap && !materialize(plan_[e - 1])) ++e;
            const int i0 = s - first;
            if (fused_) {
                lpbf_b200_opts o{phys_, 0, 0.0, Tm_, e - s, 0};
                int in_b = 0;
                const int st = lpbf_b200_advance(cur_, nxt_, &k_, plan_.data() + s, e - s, &o,
                                                 d_ring_ + i0, d_work_, work_bytes_,
                                                 this->stream(), &in_b);
                if (st != LPBF_OK)
                    throw std::runtime_error(std::string("lpbf_b200_advance: ") +
                                             lpbf_b200_status_string(st));
                if (in_b) std::swap(cur_, nxt_);
            } else {
                set_laser(plan_[s]);
                lpbf_launch_step(cur_, nxt_, &k_, phys_, this->stream());
                checkCudaErrors(cudaGetLastError());
                std::swap(cur_, nxt_);
                lpbf_launch_reduce(cur_, nx_, ny_, Tm_, d_parts_, nblk_reduce_, this->stream());
                lpbf_launch_reduce_finalize(d_parts_, nblk_reduce_, nx_, ny_, d_ring_ + i0,
                                            this->stream());
                checkCudaErrors(cudaGetLastError());
            }
            const Tick& tl = plan_[e - 1];
            if (cruise_step(tl.x_laser_csv, tl.wrapped, dom_.Lx)) {
                const int il = e - 1 - first;
                lpbf_launch_extract_col(cur_, nx_, ny_, d_ring_ + il,
                                        d_cols_ + (std::size_t)il * ny_, this->stream());
                checkCudaErrors(cudaGetLastError());
            }
            if (write_outputs_ && tl.dump) {
                auto f = std::make_shared<std::vector<double>>(N_);
                checkCudaErrors(cudaMemcpyAsync(f->data(), cur_, N_ * sizeof(double),
                                                cudaMemcpyDeviceToHost, this->stream()));
                snaps.push_back({tl.step, std::move(f)});
            }
            s = e;
        }
        const int n = last - first;
        checkCudaErrors(cudaMemcpyAsync(h_ring_, d_ring_, n * sizeof(Partial),
                                        cudaMemcpyDeviceToHost, this->stream()));
        checkCudaErrors(cudaMemcpyAsync(h_cols_, d_cols_, (std::size_t)n * ny_ * sizeof(double),
                                        cudaMemcpyDeviceToHost, this->stream()));
        checkCudaErrors(cudaStreamSynchronize(this->stream()));

        for (int i = 0; i < n; ++i) {
            const Tick& tk = plan_[first + i];
            auto m = metrics_for(tk, h_ring_[i]);
            if (m->tmax > Tm_ && cruise_step(tk.x_laser_csv, tk.wrapped, dom_.Lx))
                m->hot_col.assign(h_cols_ + (std::size_t)i * ny_, h_cols_ + (std::size_t)(i + 1) * ny_);
            this->addResult(m);
        }
        for (auto& sn : snaps) {
            auto msg = std::make_shared<SnapshotMsg>();
            msg->step = sn.step;
            msg->field = std::move(sn.field);
            this->addResult(msg);
        }
        if (last < n_steps_) this->addResult(std::make_shared<Tick>(plan_[last]));
        else done_.store(true, std::memory_order_release);
    }

    // The self-edge keeps the default rule from ever firing: finish once the
    // last step has been emitted and no Tick is queued.
    [[nodiscard]] bool canTerminate() const override {
        return done_.load(std::memory_order_acquire) && this->coreTask()->receiversEmpty();
    }

private:
    int group_cap() const {
        if (depth_ > 0) return std::min(depth_, 4);
        const long long n = (long long)nx_ * ny_;
        return n >= (1ll << 22) ? 3 : n >= (1ll << 18) ? 2 : 1;
    }
    // A step whose field must exist on the device after it (hot column on a
    // cruise step, snapshot on a dump step) ends its launch group.
    bool materialize(const Tick& t) const {
        return cruise_step(t.x_laser_csv, t.wrapped, dom_.Lx) || (write_outputs_ && t.dump);
    }
    void set_laser(const Tick& t) { k_.x_l = t.x_l; k_.y_l = t.y_l; k_.q_scale = t.q_scale; }

    std::shared_ptr<MetricsMsg> metrics_for(const Tick& tk, const Partial& g) const {
        auto m = std::make_shared<MetricsMsg>();
        m->step = tk.step;
        m->t = tk.t;
        m->x_laser_csv = tk.x_laser_csv;
        m->wrapped = tk.wrapped;
        m->dump = tk.dump;
        m->tmax = g.tmax;
        m->x_hot = static_cast<int>(g.arg % nx_);
        m->ymin = g.ymin;
        m->ymax = g.ymax;
        return m;
    }

    // Modes 0 and 1: one step, per-block partials finalized on the host.
    void per_step(const Tick& tk, bool gated) {
        set_laser(tk);
        lpbf_launch_step(cur_, nxt_, &k_, phys_, this->stream());
        checkCudaErrors(cudaGetLastError());
        std::swap(cur_, nxt_);
        lpbf_launch_reduce(cur_, nx_, ny_, Tm_, d_parts_, nblk_reduce_, this->stream());
        checkCudaErrors(cudaGetLastError());
        checkCudaErrors(cudaMemcpyAsync(parts_store_.data(), d_parts_,
                                        nblk_reduce_ * sizeof(Partial),
                                        cudaMemcpyDeviceToHost, this->stream()));
        checkCudaErrors(cudaStreamSynchronize(this->stream()));
        Partial g{-1.0, (long long)N_, ny_, -1};
        for (const Partial& q : parts_store_) {
            if (q.tmax > g.tmax || (q.tmax == g.tmax && q.arg < g.arg)) { g.tmax = q.tmax; g.arg = q.arg; }
            g.ymin = std::min(g.ymin, q.ymin);
            g.ymax = std::max(g.ymax, q.ymax);
        }
        auto m = metrics_for(tk, g);
        if (g.tmax > Tm_ && (!gated || cruise_step(tk.x_laser_csv, tk.wrapped, dom_.Lx))) {
            m->hot_col.resize(ny_);
            checkCudaErrors(cudaMemcpy2DAsync(m->hot_col.data(), sizeof(double), cur_ + m->x_hot,
                                              (std::size_t)nx_ * sizeof(double), sizeof(double),
                                              ny_, cudaMemcpyDeviceToHost, this->stream()));
            checkCudaErrors(cudaStreamSynchronize(this->stream()));
        }
        this->addResult(m);
        if (write_outputs_ && tk.dump) {
            auto f = std::make_shared<std::vector<double>>(N_);
            checkCudaErrors(cudaMemcpyAsync(f->data(), cur_, N_ * sizeof(double),
                                            cudaMemcpyDeviceToHost, this->stream()));
            checkCudaErrors(cudaStreamSynchronize(this->stream()));
            auto msg = std::make_shared<SnapshotMsg>();
            msg->step = tk.step;
            msg->field = std::move(f);
            this->addResult(msg);
        }
        if (tk.step + 1 < n_steps_) this->addResult(std::make_shared<Tick>(plan_[tk.step + 1]));
        else done_.store(true, std::memory_order_release);
    }

    Domain dom_;
    StepConst k_;
    int phys_;
    double Tm_;
    int n_steps_;
    std::vector<Tick> plan_;
    double Tamb_;
    bool write_outputs_;
    int batch_;
    int mode_;
    bool fused_;
    bool pinned_;
    int depth_ = 0;

    int nx_ = 0, ny_ = 0, nblk_reduce_ = 0, nblk_fused_ = 0;
    std::size_t N_ = 0;
    double *d_a_ = nullptr, *d_b_ = nullptr, *cur_ = nullptr, *nxt_ = nullptr;
    Partial* d_parts_ = nullptr;
    Partial* d_ring_ = nullptr;
    double* d_cols_ = nullptr;
    void* d_work_ = nullptr;
    std::size_t work_bytes_ = 0;
    Partial* h_ring_ = nullptr;
    double* h_cols_ = nullptr;
    std::vector<Partial> ring_store_, parts_store_;
    std::vector<double> cols_store_;
    std::atomic<bool> done_{false};
};

// Per-step metrics in step order: melt widths, running maxima, metrics.csv.
class MetricsTask : public hh::AbstractTask<1, MetricsMsg, StepResult> {
public:
    MetricsTask(Domain dom, double Tm, std::shared_ptr<RunAccum> acc, bool write_outputs,
                std::string snap_dir)
        : hh::AbstractTask<1, MetricsMsg, StepResult>("Metrics", 1), dom_(dom), Tm_(Tm),
          acc_(std::move(acc)), write_(write_outputs), dir_(std::move(snap_dir)) {}

    void initialize() override {
        if (!write_) return;
        csv_.open(dir_ + "/metrics.csv");
        csv_ << "step,t_us,x_laser_um,peakT_K,W_um\n";
    }

    // Linear interpolation of the two T = Tm crossings along one column.
    static double sub_grid_width_um(const std::vector<double>& col, double dy, double Tm) {
        const int n = static_cast<int>(col.size());
        int a = -1, b = -1;
        for (int y = 0; y < n; ++y)
            if (col[y] > Tm) { if (a < 0) a = y; b = y; }
        if (a < 0) return 0.0;
        double lo = a * dy, hi = b * dy;
        if (a > 0) lo = ((a - 1) + (Tm - col[a - 1]) / (col[a] - col[a - 1])) * dy;
        if (b < n - 1) hi = (b + (Tm - col[b]) / (col[b + 1] - col[b])) * dy;
        return (hi - lo) * 1e6;
    }

    void execute(std::shared_ptr<MetricsMsg> m) override {
        const double dy = dom_.dy();
        const double W = (m->ymax < 0) ? 0.0 : (m->ymax - m->ymin + 1) * dy * 1e6;
        const double Wsub = (m->tmax > Tm_ && !m->hot_col.empty())
                          ? sub_grid_width_um(m->hot_col, dy, Tm_) : 0.0;
        acc_->peak_T = std::max(acc_->peak_T, m->tmax);
        acc_->peak_W = std::max(acc_->peak_W, W);
        if (cruise_step(m->x_laser_csv, m->wrapped, dom_.Lx))
            acc_->steady_W_sub = std::max(acc_->steady_W_sub, Wsub);
        acc_->steps_seen++;
        if (write_ && m->dump)
            csv_ << m->step << ',' << m->t * 1e6 << ',' << m->x_laser_csv * 1e6 << ','
                 << m->tmax << ',' << W << '\n';
        this->addResult(std::make_shared<StepResult>(StepResult{m->step}));
    }

    void shutdown() override { if (csv_.is_open()) csv_.close(); }

private:
    Domain dom_;
    double Tm_;
    std::shared_ptr<RunAccum> acc_;
    bool write_;
    std::string dir_;
    std::ofstream csv_;
};

// Raw field snapshots, written off the GPU's critical path.
class SnapshotWriterTask : public hh::AbstractTask<1, SnapshotMsg, StepResult> {
public:
    SnapshotWriterTask(std::size_t n_threads, std::string snap_dir)
        : hh::AbstractTask<1, SnapshotMsg, StepResult>("SnapshotWriter", n_threads),
          dir_(std::move(snap_dir)) {}

    void execute(std::shared_ptr<SnapshotMsg> s) override {
        char name[64];
        std::snprintf(name, sizeof(name), "/T_step_%06d.bin", s->step);
        std::ofstream out(dir_ + name, std::ios::binary);
        out.write(reinterpret_cast<const char*>(s->field->data()),
                  static_cast<std::streamsize>(s->field->size() * sizeof(double)));
        this->addResult(std::make_shared<StepResult>(StepResult{s->step}));
    }

    std::shared_ptr<hh::AbstractTask<1, SnapshotMsg, StepResult>> copy() override {
        return std::make_shared<SnapshotWriterTask>(this->numberThreads(), dir_);
    }

private:
    std::string dir_;
};

}  // namespace lpbf

// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// hh-compat: a small stand-in for the subset of the usnistgov/hedgehog task
// graph API that hedgehog_lpbf's drivers and tasks use.  The real library is
// fetched from GitHub at configure time by the reference build and is not
// available offline, so this header lets the same task classes compile and
// run.  It is written from the call sites alone:
//
//   hh::AbstractTask<1, In, Outs...>      include/step_task.hpp:37-52,208-213
//   hh::AbstractCUDATask<1, In, Outs...>  include/gpu_step_task.hpp:53-122,322
//   hh::Graph<1, In, Outs...>             src/main.cpp:261-266,328-335,404-413
//                                         src/gpu/hh_gpu_main.cpp:339-376
//
// Semantics provided:
//   * every task has one input type and any number of output types;
//   * a task with n threads runs n instances (the original plus copy()s);
//   * addResult(x) forwards x to every receiver whose input type matches and,
//     for graph outputs, to the graph's result queue;
//   * a task terminates once canTerminate() is true; the default is "every
//     sender has terminated and the input queue is empty";
//   * graph.getBlockingResult() returns an empty optional once every output
//     task has terminated and the result queue is drained.
// No scheduling policy beyond FIFO queues and one thread per task instance.
// ---------------------------------------------------------------------------
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <variant>
#include <vector>

#ifdef HH_USE_CUDA
#include <cuda_runtime.h>
// CUDA error check used by CUDA tasks; aborts with the failing expression.
#define checkCudaErrors(val) ::hh::detail::checkCuda((val), #val, __FILE__, __LINE__)
#endif

namespace hh {

enum class ColorScheme { NONE, EXECUTION, WAIT };
enum class StructureOptions { NONE, THREADING, QUEUE, ALL };

namespace detail {

// Type-erased view of a node, enough for the graph to start, stop and link it.
class NodeBase {
public:
    virtual ~NodeBase() = default;
    virtual void start() = 0;
    virtual void join() = 0;
    virtual void addSender() = 0;
    virtual void senderTerminated() = 0;
    virtual bool terminated() const = 0;
    virtual std::string nodeName() const = 0;
    virtual std::size_t threads() const = 0;
    std::vector<NodeBase*> receivers_;   // for termination propagation
    std::vector<std::function<void()>> on_terminate_;
};

}  // namespace detail

template <std::size_t Sep, class In, class... Outs>
class AbstractTask;

namespace detail {

// State shared by every instance (thread) of one task.
template <class In, class... Outs>
class TaskCore : public NodeBase {
public:
    using Instance = AbstractTask<1, In, Outs...>;

    explicit TaskCore(Instance* root) : root_(root) {}

    template <class O>
    static constexpr bool emits() { return (std::is_same_v<O, Outs> || ...); }

    void push(std::shared_ptr<In> x) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(x));
        }
        cv_.notify_one();
    }
    bool receiversEmpty() const {
        std::lock_guard<std::mutex> lk(mu_);
        return q_.empty();
    }
    bool defaultCanTerminate() const {
        std::lock_guard<std::mutex> lk(mu_);
        return q_.empty() && live_senders_ == 0;
    }
    void addSender() override {
        std::lock_guard<std::mutex> lk(mu_);
        ++live_senders_;
    }
    void senderTerminated() override {
        {
            std::lock_guard<std::mutex> lk(mu_);
            --live_senders_;
        }
        cv_.notify_all();
    }
    void wake() { cv_.notify_all(); }
    bool terminated() const override { return done_.load(); }
    std::string nodeName() const override;
    std::size_t threads() const override;

    template <class O>
    void addReceiver(std::function<void(std::shared_ptr<O>)> f) {
        std::get<std::vector<std::function<void(std::shared_ptr<O>)>>>(routes_)
            .push_back(std::move(f));
    }
    template <class O>
    void emit(std::shared_ptr<O> x) {
        for (auto& f : std::get<std::vector<std::function<void(std::shared_ptr<O>)>>>(routes_))
            f(x);
    }

    void start() override;
    void join() override {
        for (auto& t : workers_) if (t.joinable()) t.join();
    }

private:
    void run(Instance* inst);

    Instance* root_;
    std::vector<std::shared_ptr<Instance>> copies_;
    std::vector<std::thread> workers_;
    mutable std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<In>> q_;
    int live_senders_ = 0;
    std::atomic<int> running_{0};
    std::atomic<bool> done_{false};
    std::tuple<std::vector<std::function<void(std::shared_ptr<Outs>)>>...> routes_;
};

}  // namespace detail

// ---------------------------------------------------------------------------
template <std::size_t Sep, class In, class... Outs>
class AbstractTask {
    static_assert(Sep == 1, "hh-compat supports exactly one input type");
public:
    using Core = detail::TaskCore<In, Outs...>;

    AbstractTask(std::string name, std::size_t numberThreads = 1)
        : name_(std::move(name)), nthreads_(numberThreads < 1 ? 1 : numberThreads),
          core_(std::make_shared<Core>(this)) {}
    virtual ~AbstractTask() = default;

    virtual void execute(std::shared_ptr<In>) = 0;
    virtual void initialize() {}
    virtual void shutdown() {}
    virtual bool canTerminate() const { return core_->defaultCanTerminate(); }
    virtual std::shared_ptr<AbstractTask<1, In, Outs...>> copy() { return nullptr; }

    template <class O>
    void addResult(std::shared_ptr<O> x) { core_->template emit<O>(std::move(x)); }

    std::string const& name() const { return name_; }
    std::size_t numberThreads() const { return nthreads_; }
    Core* coreTask() const { return core_.get(); }
    std::shared_ptr<Core> sharedCore() const { return core_; }
    void adoptCore(std::shared_ptr<Core> c) { core_ = std::move(c); }

private:
    std::string name_;
    std::size_t nthreads_;
    std::shared_ptr<Core> core_;
};

namespace detail {

template <class In, class... Outs>
std::string TaskCore<In, Outs...>::nodeName() const { return root_->name(); }
template <class In, class... Outs>
std::size_t TaskCore<In, Outs...>::threads() const { return root_->numberThreads(); }

template <class In, class... Outs>
void TaskCore<In, Outs...>::start() {
    const std::size_t n = root_->numberThreads();
    std::vector<Instance*> insts{root_};
    for (std::size_t i = 1; i < n; ++i) {
        auto c = root_->copy();
        if (!c) {
            std::fprintf(stderr, "hh-compat: task '%s' has %zu threads but no copy()\n",
                         root_->name().c_str(), n);
            std::abort();
        }
        c->adoptCore(root_->sharedCore());
        copies_.push_back(c);
        insts.push_back(c.get());
    }
    running_ = static_cast<int>(n);
    for (auto* inst : insts) workers_.emplace_back([this, inst] { run(inst); });
}

template <class In, class... Outs>
void TaskCore<In, Outs...>::run(Instance* inst) {
    inst->initialize();
    for (;;) {
        std::shared_ptr<In> item;
        {
            std::unique_lock<std::mutex> lk(mu_);
            for (;;) {
                if (!q_.empty()) { item = std::move(q_.front()); q_.pop_front(); break; }
                lk.unlock();
                const bool stop = inst->canTerminate();
                lk.lock();
                if (stop && q_.empty()) break;
                cv_.wait_for(lk, std::chrono::milliseconds(2));
            }
        }
        if (!item) break;
        inst->execute(std::move(item));
        cv_.notify_all();
    }
    inst->shutdown();
    if (--running_ == 0) {
        done_ = true;
        for (auto* r : receivers_) r->senderTerminated();
        for (auto& f : on_terminate_) f();
    }
    cv_.notify_all();
}

}  // namespace detail

// ---------------------------------------------------------------------------
#ifdef HH_USE_CUDA
namespace detail {
inline void checkCuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "hh-compat: %s failed at %s:%d: %s\n", what, file, line,
                     cudaGetErrorString(e));
        std::abort();
    }
}
}  // namespace detail

template <std::size_t Sep, class In, class... Outs>
class AbstractCUDATask : public AbstractTask<Sep, In, Outs...> {
public:
    AbstractCUDATask(std::string name, std::size_t numberThreads = 1)
        : AbstractTask<Sep, In, Outs...>(std::move(name), numberThreads) {}
    virtual void initializeCuda() {}
    virtual void shutdownCuda() {}
    void initialize() final {
        checkCudaErrors(cudaSetDevice(device_));
        checkCudaErrors(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        initializeCuda();
    }
    void shutdown() final {
        shutdownCuda();
        if (stream_) cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }
    cudaStream_t stream() const { return stream_; }
    int deviceId() const { return device_; }
    void deviceId(int d) { device_ = d; }

private:
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
};
#endif

// ---------------------------------------------------------------------------
template <std::size_t Sep, class In, class... Outs>
class Graph {
    static_assert(Sep == 1, "hh-compat supports exactly one graph input type");
public:
    using Result = std::variant<std::shared_ptr<Outs>...>;

    explicit Graph(std::string name) : name_(std::move(name)) {}
    ~Graph() { waitForTermination(); }

    // Graph input feeds `task`; the graph counts as one of its senders.
    template <class Task>
    void inputs(std::shared_ptr<Task> task) {
        auto core = task->sharedCore();
        core->addSender();
        remember(task, core.get());
        input_sinks_.push_back([core](std::shared_ptr<In> x) { core->push(std::move(x)); });
        input_nodes_.push_back(core.get());
    }

    // Every output of `task` whose type is a graph output type reaches the
    // result queue.
    template <class Task>
    void outputs(std::shared_ptr<Task> task) {
        auto core = task->sharedCore();
        remember(task, core.get());
        ++live_outputs_;
        attachOutputs(core, static_cast<std::tuple<Outs...>*>(nullptr));
        core->on_terminate_.push_back([this] {
            {
                std::lock_guard<std::mutex> lk(rmu_);
                --live_outputs_;
            }
            rcv_.notify_all();
        });
    }

    // Connect every output type of `from` that `to` accepts as input.
    template <class From, class To>
    void edges(std::shared_ptr<From> from, std::shared_ptr<To> to) {
        auto fc = from->sharedCore();
        auto tc = to->sharedCore();
        remember(from, fc.get());
        remember(to, tc.get());
        connect(fc, tc);
        edge_list_.push_back({fc->nodeName(), tc->nodeName()});
    }

    void executeGraph() {
        for (auto* n : nodes_) n->start();
    }
    void pushData(std::shared_ptr<In> x) {
        for (auto& s : input_sinks_) s(x);
    }
    void finishPushingData() {
        if (finished_) return;
        finished_ = true;
        for (auto* n : input_nodes_) n->senderTerminated();
    }
    std::optional<Result> getBlockingResult() {
        std::unique_lock<std::mutex> lk(rmu_);
        rcv_.wait(lk, [this] { return !results_.empty() || live_outputs_ == 0; });
        if (results_.empty()) return std::nullopt;
        Result r = std::move(results_.front());
        results_.pop_front();
        return r;
    }
    void waitForTermination() {
        finishPushingData();
        for (auto* n : nodes_) n->join();
    }
    void createDotFile(std::string const& path, ColorScheme = ColorScheme::NONE,
                       StructureOptions = StructureOptions::NONE) const {
        std::ofstream f(path);
        f << "digraph \"" << name_ << "\" {\n";
        for (auto* n : nodes_)
            f << "  \"" << n->nodeName() << "\" [label=\"" << n->nodeName()
              << "\\nthreads: " << n->threads() << "\"];\n";
        for (auto& e : edge_list_)
            f << "  \"" << e.first << "\" -> \"" << e.second << "\";\n";
        f << "}\n";
    }

private:
    template <class Task>
    void remember(std::shared_ptr<Task> const& t, detail::NodeBase* n) {
        for (auto* m : nodes_) if (m == n) return;
        nodes_.push_back(n);
        owners_.push_back(std::static_pointer_cast<void>(t));
    }

    template <class Core, class... Os>
    void attachOutputs(std::shared_ptr<Core> const& core, std::tuple<Os...>*) {
        (attachOne<Core, Os>(core), ...);
    }
    template <class Core, class O>
    void attachOne(std::shared_ptr<Core> const& core) {
        if constexpr (canEmit<Core, O>()) {
            core->template addReceiver<O>([this](std::shared_ptr<O> x) {
                {
                    std::lock_guard<std::mutex> lk(rmu_);
                    results_.emplace_back(Result{std::move(x)});
                }
                rcv_.notify_all();
            });
        }
    }
    template <class Core, class O>
    static constexpr bool canEmit() { return Core::template emits<O>(); }

    template <class FromCore, class ToIn, class... ToOuts>
    void connect(std::shared_ptr<FromCore> const& fc,
                 std::shared_ptr<detail::TaskCore<ToIn, ToOuts...>> const& tc) {
        static_assert(FromCore::template emits<ToIn>(),
                      "hh-compat edge: sender does not produce the receiver's input type");
        auto keep = tc;
        fc->template addReceiver<ToIn>([keep](std::shared_ptr<ToIn> x) { keep->push(std::move(x)); });
        if (static_cast<detail::NodeBase*>(fc.get()) != static_cast<detail::NodeBase*>(tc.get())) {
            tc->addSender();
            fc->receivers_.push_back(tc.get());
        } else {
            self_edges_.push_back(tc.get());
        }
    }

    std::string name_;
    std::vector<detail::NodeBase*> nodes_;
    std::vector<std::shared_ptr<void>> owners_;
    std::vector<std::function<void(std::shared_ptr<In>)>> input_sinks_;
    std::vector<detail::NodeBase*> input_nodes_;
    std::vector<std::pair<std::string, std::string>> edge_list_;
    std::vector<detail::NodeBase*> self_edges_;
    bool finished_ = false;
    std::mutex rmu_;
    std::condition_variable rcv_;
    std::deque<Result> results_;
    int live_outputs_ = 0;
};

}  // namespace hh

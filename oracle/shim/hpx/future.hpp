// Test infrastructure (oracle build only): a minimal task runtime that offers
// the subset of the HPX API used by GPRat's CPU sources, so that those
// sources compile unmodified without HPX.  Nothing in the product links it.
//
// Provided: hpx::shared_future / hpx::future, hpx::async, hpx::dataflow,
// hpx::unwrapping, hpx::annotated_function, hpx::make_ready_future,
// hpx::wait_all, hpx::start / stop / post / finalize / suspend / resume.
//
// Design: a fixed pool of std::threads with one FIFO queue.  A dataflow task
// counts its unready futures and is queued when the last one becomes ready
// (continuations, no blocking).  A pool thread that calls get() on an unready
// future executes queued tasks while it waits, so nested waits cannot starve
// the pool.  The pool size is taken from "--hpx:threads=N" passed to
// hpx::start (default: hardware concurrency).
#pragma once

#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <exception>
#include <functional>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <numeric>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace hpx
{
namespace shim
{

class pool
{
  public:
    static pool &instance()
    {
        static pool p;
        return p;
    }

    void ensure_started(unsigned n = 0)
    {
        std::lock_guard<std::mutex> lk(start_mtx_);
        if (!workers_.empty())
        {
            return;
        }
        if (n == 0)
        {
            n = requested_ ? requested_ : std::max(1u, std::thread::hardware_concurrency());
        }
        stopping_ = false;
        for (unsigned i = 0; i < n; ++i)
        {
            workers_.emplace_back([this] { worker_loop(); });
        }
    }

    void request_threads(unsigned n) { requested_ = n; }

    void submit(std::function<void()> task)
    {
        ensure_started();
        {
            std::lock_guard<std::mutex> lk(q_mtx_);
            queue_.push_back(std::move(task));
        }
        q_cv_.notify_one();
    }

    // Runs one queued task on the calling thread; returns false if none.
    bool run_one()
    {
        std::function<void()> task;
        {
            std::lock_guard<std::mutex> lk(q_mtx_);
            if (queue_.empty())
            {
                return false;
            }
            task = std::move(queue_.front());
            queue_.pop_front();
        }
        task();
        return true;
    }

    static bool on_worker() { return worker_flag(); }

    void shutdown()
    {
        {
            std::lock_guard<std::mutex> lk(q_mtx_);
            stopping_ = true;
        }
        q_cv_.notify_all();
        std::lock_guard<std::mutex> lk(start_mtx_);
        for (auto &t : workers_)
        {
            if (t.joinable())
            {
                t.join();
            }
        }
        workers_.clear();
    }

    ~pool() { shutdown(); }

  private:
    static bool &worker_flag()
    {
        static thread_local bool flag = false;
        return flag;
    }

    void worker_loop()
    {
        worker_flag() = true;
        for (;;)
        {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> lk(q_mtx_);
                q_cv_.wait(lk, [this] { return stopping_ || !queue_.empty(); });
                if (queue_.empty())
                {
                    return;  // stopping and drained
                }
                task = std::move(queue_.front());
                queue_.pop_front();
            }
            task();
        }
    }

    std::mutex start_mtx_;
    std::vector<std::thread> workers_;
    std::mutex q_mtx_;
    std::condition_variable q_cv_;
    std::deque<std::function<void()>> queue_;
    bool stopping_ = false;
    unsigned requested_ = 0;
};

template <typename T>
struct state
{
    std::mutex mtx;
    std::condition_variable cv;
    bool ready = false;
    std::optional<T> value;
    std::exception_ptr error;
    std::vector<std::function<void()>> continuations;

    void fulfil(T &&v)
    {
        std::vector<std::function<void()>> conts;
        {
            std::lock_guard<std::mutex> lk(mtx);
            value.emplace(std::move(v));
            ready = true;
            conts.swap(continuations);
        }
        cv.notify_all();
        for (auto &c : conts)
        {
            c();
        }
    }

    void fail(std::exception_ptr e)
    {
        std::vector<std::function<void()>> conts;
        {
            std::lock_guard<std::mutex> lk(mtx);
            error = e;
            ready = true;
            conts.swap(continuations);
        }
        cv.notify_all();
        for (auto &c : conts)
        {
            c();
        }
    }

    // Calls c once the state is ready (immediately if it already is).
    void on_ready(std::function<void()> c)
    {
        {
            std::lock_guard<std::mutex> lk(mtx);
            if (!ready)
            {
                continuations.push_back(std::move(c));
                return;
            }
        }
        c();
    }

    void wait()
    {
        if (pool::on_worker())
        {
            for (;;)
            {
                {
                    std::lock_guard<std::mutex> lk(mtx);
                    if (ready)
                    {
                        return;
                    }
                }
                if (!pool::instance().run_one())
                {
                    std::unique_lock<std::mutex> lk(mtx);
                    cv.wait_for(lk, std::chrono::microseconds(200), [this] { return ready; });
                }
            }
        }
        std::unique_lock<std::mutex> lk(mtx);
        cv.wait(lk, [this] { return ready; });
    }
};

}  // namespace shim

template <typename T>
class shared_future
{
  public:
    using value_type = T;

    shared_future() = default;
    explicit shared_future(std::shared_ptr<shim::state<T>> s) : s_(std::move(s)) { }

    const T &get() const
    {
        if (!s_)
        {
            throw std::runtime_error("hpx shim: get() on an empty future");
        }
        s_->wait();
        if (s_->error)
        {
            std::rethrow_exception(s_->error);
        }
        return *s_->value;
    }

    void wait() const
    {
        if (s_)
        {
            s_->wait();
        }
    }

    bool valid() const { return static_cast<bool>(s_); }

    bool is_ready() const
    {
        if (!s_)
        {
            return false;
        }
        std::lock_guard<std::mutex> lk(s_->mtx);
        return s_->ready;
    }

    std::shared_ptr<shim::state<T>> state_ptr() const { return s_; }

  private:
    std::shared_ptr<shim::state<T>> s_;
};

template <typename T>
using future = shared_future<T>;

namespace shim
{

template <typename T>
struct is_future : std::false_type
{ };

template <typename T>
struct is_future<shared_future<T>> : std::true_type
{ };

template <typename T>
struct is_future_vector : std::false_type
{ };

template <typename T>
struct is_future_vector<std::vector<shared_future<T>>> : std::true_type
{ };

// Completes `out` with the result of calling `fn` (unwrapping a returned
// future, as HPX does for dataflow/async).
template <typename R, typename Fn>
struct completer
{
    static void run(const std::shared_ptr<state<R>> &out, Fn &fn)
    {
        try
        {
            out->fulfil(fn());
        }
        catch (...)
        {
            out->fail(std::current_exception());
        }
    }
};

template <typename U, typename Fn>
struct completer<shared_future<U>, Fn>
{
    static void run(const std::shared_ptr<state<U>> &out, Fn &fn)
    {
        try
        {
            shared_future<U> inner = fn();
            auto s = inner.state_ptr();
            s->on_ready(
                [out, s]
                {
                    if (s->error)
                    {
                        out->fail(s->error);
                    }
                    else
                    {
                        U copy = *s->value;
                        out->fulfil(std::move(copy));
                    }
                });
        }
        catch (...)
        {
            out->fail(std::current_exception());
        }
    }
};

template <typename R>
struct result_of_future
{
    using type = R;
};

template <typename U>
struct result_of_future<shared_future<U>>
{
    using type = U;
};

// Registers `cb` on every future contained in `arg`; `pending` counts them.
template <typename A>
void collect(A &arg, std::vector<std::function<void(std::function<void()>)>> &hooks)
{
    if constexpr (is_future<A>::value)
    {
        auto s = arg.state_ptr();
        if (s)
        {
            hooks.push_back([s](std::function<void()> cb) { s->on_ready(std::move(cb)); });
        }
    }
    else if constexpr (is_future_vector<A>::value)
    {
        for (auto &f : arg)
        {
            auto s = f.state_ptr();
            if (s)
            {
                hooks.push_back([s](std::function<void()> cb) { s->on_ready(std::move(cb)); });
            }
        }
    }
}

template <typename T>
decltype(auto) unwrap_one(T &arg)
{
    if constexpr (is_future<T>::value)
    {
        return arg.get();
    }
    else if constexpr (is_future_vector<T>::value)
    {
        using V = typename T::value_type::value_type;
        std::vector<V> out;
        out.reserve(arg.size());
        for (auto &f : arg)
        {
            out.push_back(f.get());
        }
        return out;
    }
    else
    {
        return (arg);
    }
}

}  // namespace shim

template <typename F>
std::decay_t<F> annotated_function(F &&f, const char *)
{
    return std::forward<F>(f);
}

template <typename F>
auto unwrapping(F &&f)
{
    return [fn = std::decay_t<F>(std::forward<F>(f))](auto &&...args) mutable -> decltype(auto)
    { return std::invoke(fn, shim::unwrap_one(args)...); };
}

template <typename T>
shared_future<std::decay_t<T>> make_ready_future(T &&v)
{
    auto s = std::make_shared<shim::state<std::decay_t<T>>>();
    s->fulfil(std::decay_t<T>(std::forward<T>(v)));
    return shared_future<std::decay_t<T>>(s);
}

// Runs f(args...) once every future among args (or in vectors of futures
// among args) is ready.  Futures are passed through as futures.
template <typename F, typename... Args>
auto dataflow(F &&f, Args &&...args)
{
    using Fn = std::decay_t<F>;
    using Tuple = std::tuple<std::decay_t<Args>...>;
    using Raw = std::invoke_result_t<Fn &, std::decay_t<Args> &...>;
    using R = typename shim::result_of_future<Raw>::type;

    auto out = std::make_shared<shim::state<R>>();
    auto payload = std::make_shared<std::pair<Fn, Tuple>>(Fn(std::forward<F>(f)), Tuple(std::forward<Args>(args)...));

    std::vector<std::function<void(std::function<void()>)>> hooks;
    std::apply([&hooks](auto &...a) { (shim::collect(a, hooks), ...); }, payload->second);

    auto launch = [out, payload]
    {
        shim::pool::instance().submit(
            [out, payload]
            {
                auto call = [&payload]() -> Raw { return std::apply(payload->first, payload->second); };
                shim::completer<Raw, decltype(call)>::run(out, call);
            });
    };

    if (hooks.empty())
    {
        launch();
    }
    else
    {
        auto remaining = std::make_shared<std::atomic<std::size_t>>(hooks.size());
        for (auto &h : hooks)
        {
            h(
                [remaining, launch]
                {
                    if (remaining->fetch_sub(1) == 1)
                    {
                        launch();
                    }
                });
        }
    }
    return shared_future<R>(out);
}

template <typename F, typename... Args>
auto async(F &&f, Args &&...args)
{
    return dataflow(std::forward<F>(f), std::forward<Args>(args)...);
}

template <typename... Fs>
void wait_all(const Fs &...fs)
{
    auto wait_one = [](const auto &x)
    {
        using X = std::decay_t<decltype(x)>;
        if constexpr (shim::is_future<X>::value)
        {
            x.wait();
        }
        else if constexpr (shim::is_future_vector<X>::value)
        {
            for (auto &f : x)
            {
                f.wait();
            }
        }
    };
    (wait_one(fs), ...);
}

}  // namespace hpx

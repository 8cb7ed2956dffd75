// ThreadPool.hpp — TEST INFRASTRUCTURE ONLY. Stand-in for GlassImage's
// thread pool as SURF.cpp's SURFInvoker::run uses it: every enqueued task
// runs on a thread of its own; the destructor waits for all of them.
#pragma once

#include <thread>
#include <utility>
#include <vector>

class ThreadPool {
   public:
    explicit ThreadPool(size_t) {}
    template <class F>
    void enqueue(F&& f) {
        _threads.emplace_back(std::forward<F>(f));
    }
    ~ThreadPool() {
        for (auto& t : _threads) t.join();
    }

   private:
    std::vector<std::thread> _threads;
};

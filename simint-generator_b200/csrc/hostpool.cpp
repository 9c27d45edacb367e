#include "hostpool.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace sb200 {

namespace {

struct Pool
{
    std::vector<std::thread> workers;
    std::mutex m, call_m;
    std::condition_variable cv_work, cv_done;
    const std::function<void(size_t, size_t)> * fn = nullptr;
    size_t n = 0, piece = 0, next = 0;
    int pending = 0;
    long long gen = 0;
    bool stop = false;

    Pool()
    {
        const unsigned hc = std::thread::hardware_concurrency();
        const int nw = (int)std::min<unsigned>(hc > 1 ? hc - 1 : 0, 31);
        for(int i = 0; i < nw; i++)
            workers.emplace_back([this] { run(); });
    }

    ~Pool()
    {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        cv_work.notify_all();
        for(auto & t : workers)
            t.join();
    }

    // take pieces until none are left
    void drain()
    {
        for(;;)
        {
            size_t lo;
            {
                std::lock_guard<std::mutex> lk(m);
                if(next >= n)
                    return;
                lo = next;
                next = std::min(n, next + piece);
            }
            (*fn)(lo, std::min(n, lo + piece));
        }
    }

    void run()
    {
        long long seen = 0;
        for(;;)
        {
            {
                std::unique_lock<std::mutex> lk(m);
                cv_work.wait(lk, [&] { return stop || gen != seen; });
                if(stop)
                    return;
                seen = gen;
            }
            drain();
            {
                std::lock_guard<std::mutex> lk(m);
                if(--pending == 0)
                    cv_done.notify_one();
            }
        }
    }
};

Pool & pool()
{
    static Pool p;
    return p;
}

} // namespace

void parallel_for(size_t n, size_t min_piece, const std::function<void(size_t, size_t)> & fn)
{
    Pool & p = pool();
    const size_t nthreads = p.workers.size() + 1;
    if(n == 0)
        return;
    if(p.workers.empty() || n <= min_piece)
    {
        fn(0, n);
        return;
    }
    std::lock_guard<std::mutex> call(p.call_m);
    {
        std::lock_guard<std::mutex> lk(p.m);
        p.fn = &fn;
        p.n = n;
        p.piece = std::max(min_piece, (n + 4 * nthreads - 1) / (4 * nthreads));
        p.next = 0;
        p.pending = (int)p.workers.size();
        p.gen++;
    }
    p.cv_work.notify_all();
    p.drain();
    std::unique_lock<std::mutex> lk(p.m);
    p.cv_done.wait(lk, [&] { return p.pending == 0; });
    p.fn = nullptr;
}

// 256 KB blocks, at least two per piece: a copy of a few MB already spreads
// over most host threads (one thread copies about 10 GB/s)
void parallel_copy(void * dst, const void * src, size_t bytes)
{
    const size_t blk = 256 << 10;
    parallel_for((bytes + blk - 1) / blk, 2, [&](size_t lo, size_t hi) {
        const size_t a = lo * blk, b = std::min(bytes, hi * blk);
        memcpy((char *)dst + a, (const char *)src + a, b - a);
    });
}

} // namespace sb200

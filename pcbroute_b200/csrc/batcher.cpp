// The round batcher: searches that arrive concurrently from the router's worker threads are solved together, in one
// persistent relaxation launch.
//
// pcbroute's route_waves runs T worker threads ahead of the commit point (src/router.cpp:2119-2242). Each worker that
// hands a search to the back end blocks in gpu_solve (src/router.cpp:1587), so at any moment several searches of the
// same wave are in flight. The reference back end runs them on separate streams, one sweep loop each
// (src/gpu.cu:550-622). Here every search first prepares its inputs on its own slot stream (uploads, cost
// resolution), then joins a queue. The first thread to find no launch running becomes the leader. It waits until no
// other search is still preparing (or the batching window ends) and solves everything queued in one solve_batch call.
//
// Results do not depend on the grouping. Every search has its own distance field, worklists and bound in the batch,
// and the field is the exact least fixed point, whatever the schedule.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

struct Ticket {
    BatchItem* item;
    BatchResult* res;
    bool done = false;
};

struct Batcher {
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Ticket*> queue;
    bool leading = false;          // a leader is gathering or solving
    int preparing = 0;             // searches that will submit soon
    cudaStream_t stream = nullptr;
    long long batches = 0, searches = 0;
    int window_us = 2000;          // current wait limit of a leader
    int cap_us = 2000;             // its upper limit
    bool adaptive = true;          // tune window_us from what the waits bring in
} g_b;

// The batching window tunes itself: a leader whose whole wait brought no other search in shrinks it (x0.7, down to
// 50 us), since the searches still preparing were too far from submitting; a wait that did bring searches in
// widens it (x1.25, up to the cap). A wait that ended because nobody was preparing any more leaves it as it is.
void tune_window(bool timed_out, size_t before, size_t after) {
    if (!g_b.adaptive) return;
    if (timed_out && after == before) g_b.window_us = std::max(50, int(g_b.window_us * 0.7));
    else if (after > before) g_b.window_us = std::min(g_b.cap_us, int(g_b.window_us * 1.25) + 1);
}

}  // namespace

void batcher_enter() {
    std::lock_guard<std::mutex> g(g_b.mu);
    ++g_b.preparing;
}

void batcher_leave() {
    std::lock_guard<std::mutex> g(g_b.mu);
    --g_b.preparing;
    g_b.cv.notify_all();
}

int batcher_submit(BatchItem& item, BatchResult& res) {
    Ticket t{&item, &res};
    std::unique_lock<std::mutex> lk(g_b.mu);
    --g_b.preparing;
    g_b.queue.push_back(&t);
    g_b.cv.notify_all();
    while (!t.done) {
        if (g_b.leading || g_b.queue.empty()) {
            g_b.cv.wait(lk);
            continue;
        }
        // lead: wait for the searches still preparing their inputs, at most the batching window
        g_b.leading = true;
        const size_t before = g_b.queue.size();
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(g_b.window_us);
        const bool ready = g_b.cv.wait_until(lk, until, [] { return g_b.preparing <= 0; });
        tune_window(!ready, before, g_b.queue.size());
        std::vector<Ticket*> take;
        take.swap(g_b.queue);
        if (!g_b.stream && cudaStreamCreateWithFlags(&g_b.stream, cudaStreamNonBlocking) != cudaSuccess) g_b.stream = nullptr;
        cudaStream_t s = g_b.stream;
        lk.unlock();
        std::vector<BatchItem> items(take.size());
        for (size_t k = 0; k < take.size(); ++k) items[k] = *take[k]->item;
        const int rc = s ? solve_batch(items.data(), int(items.size()), s) : -1;
        const std::string err = rc != 0 ? (s ? last_error() : std::string("batcher stream creation failed")) : std::string();
        const long long tv = last_stats().tile_visits;
        const float kms = last_stats().kernel_ms;
        lk.lock();
        for (size_t k = 0; k < take.size(); ++k) {
            *take[k]->item = items[k];
            take[k]->res->rc = rc;
            take[k]->res->error = err;
            take[k]->res->tile_visits = tv;
            take[k]->res->batch_size = int(take.size());
            take[k]->res->kernel_ms = kms;
            take[k]->done = true;
        }
        ++g_b.batches;
        g_b.searches += (long long)take.size();
        g_b.leading = false;
        g_b.cv.notify_all();
    }
    return res.rc;
}

void batcher_window(int us) {
    std::lock_guard<std::mutex> g(g_b.mu);
    if (us < 0) {           // tuned between 50 us and the cap
        g_b.adaptive = true;
        return;
    }
    g_b.adaptive = false;   // fixed
    g_b.window_us = us;
}

void batcher_stats(long long* batches, long long* searches) {
    std::lock_guard<std::mutex> g(g_b.mu);
    *batches = g_b.batches;
    *searches = g_b.searches;
}

}  // namespace pcbg

extern "C" void pcbg_batch_window(int32_t us) { pcbg::batcher_window(us); }

extern "C" void pcbg_batcher_stats(int64_t* batches, int64_t* searches) {
    long long b = 0, s = 0;
    pcbg::batcher_stats(&b, &s);
    if (batches) *batches = b;
    if (searches) *searches = s;
}

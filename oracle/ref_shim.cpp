// Test infrastructure only: fiber scheduler behind ref_shim.hpp.
#include "ref_shim.hpp"

#include <ucontext.h>

#include <atomic>
#include <cstdlib>
#include <stdexcept>
#include <thread>
#include <vector>

struct vt_fiber {
    vt_dim3 tid;
    ucontext_t ctx;
    bool done;
    bool at_barrier;
    char* stack;
};

thread_local vt_fiber* vt_cur_fiber = nullptr;
thread_local vt_dim3 vt_block_idx;
thread_local vt_dim3 vt_block_dim;
thread_local vt_dim3 vt_grid_dim;

static thread_local ucontext_t vt_sched_ctx;
static thread_local const std::function<void()>* vt_body = nullptr;

const vt_dim3& vt_thread_idx() { return vt_cur_fiber->tid; }

void __syncthreads() {
    vt_fiber* f = vt_cur_fiber;
    f->at_barrier = true;
    swapcontext(&f->ctx, &vt_sched_ctx);
}

static void vt_trampoline() {
    (*vt_body)();
    vt_cur_fiber->done = true;
    swapcontext(&vt_cur_fiber->ctx, &vt_sched_ctx);
}

static const size_t kStack = 256 * 1024;

static void vt_run_block(std::vector<vt_fiber>& fibers) {
    for (auto& f : fibers) {
        f.done = false;
        f.at_barrier = false;
        getcontext(&f.ctx);
        f.ctx.uc_stack.ss_sp = f.stack;
        f.ctx.uc_stack.ss_size = kStack;
        f.ctx.uc_link = nullptr;
        makecontext(&f.ctx, vt_trampoline, 0);
    }
    for (;;) {
        bool any_live = false;
        for (auto& f : fibers) {
            if (f.done) continue;
            any_live = true;
            vt_cur_fiber = &f;
            swapcontext(&vt_sched_ctx, &f.ctx);
        }
        if (!any_live) break;
        // every live fiber is now at the barrier (or finished): release it
        for (auto& f : fibers) f.at_barrier = false;
    }
}

void vt_launch(vt_dim3 grid, vt_dim3 block, const std::function<void()>& body, int os_threads) {
    const long nblocks = (long)grid.x * grid.y * grid.z;
    const unsigned nthr = block.x * block.y * block.z;
    if (nblocks <= 0 || nthr == 0) return;
    int nos = os_threads > 0 ? os_threads : (int)std::thread::hardware_concurrency();
    if (nos < 1) nos = 1;
    if (nos > nblocks) nos = (int)nblocks;
    std::atomic<long> next(0);
    auto worker = [&]() {
        vt_body = &body;
        vt_grid_dim = grid;
        vt_block_dim = block;
        std::vector<vt_fiber> fibers(nthr);
        for (unsigned t = 0; t < nthr; ++t) {
            fibers[t].stack = (char*)std::malloc(kStack);
            if (!fibers[t].stack) throw std::runtime_error("fiber stack");
            fibers[t].tid.x = t % block.x;
            fibers[t].tid.y = (t / block.x) % block.y;
            fibers[t].tid.z = t / (block.x * block.y);
        }
        for (;;) {
            long b = next.fetch_add(1);
            if (b >= nblocks) break;
            vt_block_idx.x = (unsigned)(b % grid.x);
            vt_block_idx.y = (unsigned)((b / grid.x) % grid.y);
            vt_block_idx.z = (unsigned)(b / ((long)grid.x * grid.y));
            vt_run_block(fibers);
        }
        for (auto& f : fibers) std::free(f.stack);
    };
    if (nos == 1) {
        worker();
        return;
    }
    std::vector<std::thread> pool;
    for (int i = 0; i < nos; ++i) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
}

// pearl_batch.cu — host side of batched instances: creation, group
// assignment, autotuning and the batch C ABI (the kernel is pearl_batch_kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include "pearl_host.hpp"

using namespace pearl_gpu;

// ============================================================ batched instances
struct pearl_gpu_batch {
    int device = 0, n = 0;
    std::vector<pearl_gpu_ctx*> inst;  // host bookkeeping and buffers of every instance
    Ctl* d_ctls = nullptr;             // the instances' control blocks, contiguous
    Ctl* h_ctls = nullptr;             // pinned mirror
    BatchInstance* d_inst = nullptr;
    int* d_order = nullptr;
    int* d_first = nullptr;
    int* d_block_group = nullptr;
    int* d_group_block0 = nullptr;
    Ctl* d_group_ctl = nullptr;
    double* d_group_part = nullptr;
    int per_sm = 0, sms = 0, grid = 0, group_blocks = 0, ngroups = 0;  // group_blocks -1: sized per instance
    double pass_overhead_tiles = 4;  // sized groups: fixed cost of a pass, in tiles of one block
    bool use_tma = true;      // TMA staging in use (needs the 32x16 tile)
    bool tma_capable = true;  // tensor maps of every instance encoded and the shared memory granted
    int tile_wx = 0;          // tile shape of every instance: 2^tile_wx warps side by side in x
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0;
    long long launches = 0;
    std::string error;
};

namespace {

int bfail(pearl_gpu_batch* b, int status, const std::string& msg) {
    if (b) b->error = msg;
    return status;
}
#define PB_CUDA(b, call)                                                                        \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return bfail(b, PEARL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Assignment of instances to groups.  A pass over an instance of T tiles on a
// group of g blocks takes about `o + ceil(T/g)` tile times (o: the pass's
// fixed cost, grid barrier and pipeline fill, in tiles of one block), and a
// group runs its instances one after another.  Instances go longest first to
// the group where they would finish earliest (groups of one size are
// interchangeable, so a min-heap per size suffices).  Returns the longest
// group time; fills lists[g] when lists is given.
double earliest_finish(const std::vector<long long>& tiles, const std::vector<int>& sizes, double o,
                       std::vector<std::vector<int>>* lists) {
    using Slot = std::pair<double, int>;  // (time so far, group)
    std::vector<int> distinct;
    for (int g : sizes)
        if (std::find(distinct.begin(), distinct.end(), g) == distinct.end()) distinct.push_back(g);
    std::sort(distinct.begin(), distinct.end());
    std::vector<std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>>> heaps(distinct.size());
    for (int j = 0; j < (int)sizes.size(); ++j)
        heaps[std::lower_bound(distinct.begin(), distinct.end(), sizes[j]) - distinct.begin()].push({0.0, j});
    std::vector<int> idx(tiles.size());
    for (int i = 0; i < (int)idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return tiles[x] > tiles[y]; });
    if (lists) lists->assign(sizes.size(), {});
    double longest = 0;
    for (int i : idx) {
        int best = -1;
        double finish = 0;
        for (size_t k = 0; k < distinct.size(); ++k) {
            if (heaps[k].empty()) continue;
            const double f = heaps[k].top().first + o + (double)((tiles[i] + distinct[k] - 1) / distinct[k]);
            if (best < 0 || f < finish) {
                best = (int)k;
                finish = f;
            }
        }
        const Slot top = heaps[best].top();
        heaps[best].pop();
        heaps[best].push({finish, top.second});
        if (lists) (*lists)[top.second].push_back(i);
        longest = std::max(longest, finish);
    }
    return longest;
}

// Longest modelled group time of a given assignment.
double earliest_finish_on(const std::vector<long long>& tiles, const std::vector<int>& sizes,
                          const std::vector<std::vector<int>>& lists, double o) {
    double longest = 0;
    for (size_t g = 0; g < sizes.size(); ++g) {
        double t = 0;
        for (int i : lists[g]) t += o + (double)((tiles[i] + sizes[g] - 1) / sizes[g]);
        longest = std::max(longest, t);
    }
    return longest;
}

// Group sizes for PEARL_BATCH_SIZED_GROUPS: compositions of groups of s, 2s
// and 4s blocks (s = 1, 2, 4, .. up to the grid) filling the grid, and one
// group of floor(grid / n) blocks per instance (for a single instance: the
// whole grid), each scored by earliest_finish; the shortest wins.  Groups left
// without an instance are dropped.  Returns the sizes and fills lists.
std::vector<int> sized_groups(const std::vector<long long>& tiles, int max_grid, double o,
                              std::vector<std::vector<int>>& lists) {
    std::vector<int> best;
    double best_t = 0;
    const int n = (int)tiles.size();
    if (n <= max_grid) {
        best.assign(n, max_grid / n);
        best_t = earliest_finish(tiles, best, o, nullptr);
    }
    for (int s = 1; s <= max_grid; s *= 2) {
        const int big = 4 * s, mid = 2 * s;
        const int step_big = std::max(1, max_grid / big / 32), step_mid = std::max(1, max_grid / mid / 32);
        for (int nb = 0; nb * big <= max_grid; nb += step_big)
            for (int nm = 0; nb * big + nm * mid <= max_grid; nm += step_mid) {
                const int ns = (max_grid - nb * big - nm * mid) / s;
                std::vector<int> sizes;
                sizes.insert(sizes.end(), nb, big);
                sizes.insert(sizes.end(), nm, mid);
                sizes.insert(sizes.end(), ns, s);
                if (sizes.empty()) continue;
                const double t = earliest_finish(tiles, sizes, o, nullptr);
                if (best.empty() || t < best_t) {
                    best_t = t;
                    best = sizes;
                }
            }
    }
    std::vector<std::vector<int>> all;
    earliest_finish(tiles, best, o, &all);
    std::vector<int> sizes;
    lists.clear();
    for (size_t g = 0; g < best.size(); ++g)
        if (!all[g].empty()) {
            sizes.push_back(best[g]);
            lists.push_back(all[g]);
        }
    return sizes;
}

// The groups of a launch of `max_grid` blocks: gb blocks each, or the sizes
// sized_groups picks for gb = PEARL_BATCH_SIZED_GROUPS, instances assigned by
// earliest_finish.  Returns the modelled longest group time.
double plan_groups(const std::vector<long long>& tiles, int max_grid, int gb, double o, std::vector<int>& sizes,
                   std::vector<std::vector<int>>& lists) {
    if (gb == PEARL_BATCH_SIZED_GROUPS) {
        sizes = sized_groups(tiles, max_grid, o, lists);
        return earliest_finish_on(tiles, sizes, lists, o);
    }
    sizes.assign(max_grid / gb, gb);
    return earliest_finish(tiles, sizes, o, &lists);
}

// Give every instance the tile shape `wx` and split the cooperative grid into
// groups, of `gb` blocks each or, for gb = PEARL_BATCH_SIZED_GROUPS, of the
// sizes sized_groups picks, with instances assigned by earliest_finish.  Only
// a group's size bears on an instance's arithmetic (which block owns which
// tile), not which group it is in.  TMA staging needs the 32x16 tile.
int batch_configure(pearl_gpu_batch* b, int gb, bool use_tma, int wx) {
    const int max_grid = b->per_sm * b->sms;
    if (gb != PEARL_BATCH_SIZED_GROUPS && (gb < 1 || gb > max_grid))
        return bfail(b, PEARL_ERR_INVALID_ARGUMENT, "invalid group size");
    if (wx < 0 || wx > 3) return bfail(b, PEARL_ERR_INVALID_ARGUMENT, "invalid tile shape");
    b->group_blocks = gb;
    b->tile_wx = wx;
    b->use_tma = use_tma && wx == 0 && b->tma_capable;
    for (auto* c : b->inst) set_tile_shape(c, wx);
    std::vector<long long> tiles(b->n);
    for (int i = 0; i < b->n; ++i) tiles[i] = b->inst[i]->P.ntiles;
    std::vector<int> sizes;                // blocks of each group
    std::vector<std::vector<int>> lists;  // instances of each group
    plan_groups(tiles, max_grid, gb, b->pass_overhead_tiles, sizes, lists);
    b->ngroups = (int)sizes.size();
    std::vector<int> order, first(1, 0), block_group, group_block0(1, 0);
    for (int g = 0; g < b->ngroups; ++g) {
        order.insert(order.end(), lists[g].begin(), lists[g].end());
        first.push_back((int)order.size());
        block_group.insert(block_group.end(), sizes[g], g);
        group_block0.push_back((int)block_group.size());
    }
    b->grid = (int)block_group.size();
    cudaFree(b->d_order);
    cudaFree(b->d_first);
    cudaFree(b->d_block_group);
    cudaFree(b->d_group_block0);
    cudaFree(b->d_group_ctl);
    cudaFree(b->d_group_part);
    b->d_order = nullptr;
    b->d_first = nullptr;
    b->d_block_group = nullptr;
    b->d_group_block0 = nullptr;
    b->d_group_ctl = nullptr;
    b->d_group_part = nullptr;
    PB_CUDA(b, cudaMalloc(&b->d_order, sizeof(int) * std::max(1, b->n)));
    PB_CUDA(b, cudaMalloc(&b->d_first, sizeof(int) * first.size()));
    PB_CUDA(b, cudaMalloc(&b->d_block_group, sizeof(int) * block_group.size()));
    PB_CUDA(b, cudaMalloc(&b->d_group_block0, sizeof(int) * group_block0.size()));
    PB_CUDA(b, cudaMalloc(&b->d_group_ctl, sizeof(Ctl) * b->ngroups));
    PB_CUDA(b, cudaMalloc(&b->d_group_part, sizeof(double) * (size_t)b->grid * 2 * kMaxRed));
    PB_CUDA(b, cudaMemcpy(b->d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
    PB_CUDA(b, cudaMemcpy(b->d_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
    PB_CUDA(b, cudaMemcpy(b->d_block_group, block_group.data(), sizeof(int) * block_group.size(),
                          cudaMemcpyHostToDevice));
    PB_CUDA(b, cudaMemcpy(b->d_group_block0, group_block0.data(), sizeof(int) * group_block0.size(),
                          cudaMemcpyHostToDevice));
    PB_CUDA(b, cudaMemset(b->d_group_ctl, 0, sizeof(Ctl) * b->ngroups));
    // per-instance descriptors (tensor maps, parameters, buffers)
    std::vector<BatchInstance> hi(b->n);
    for (int i = 0; i < b->n; ++i) {
        std::memcpy(hi[i].maps, b->inst[i]->maps, sizeof hi[i].maps);
        hi[i].P = b->inst[i]->P;
        hi[i].B = b->inst[i]->B;
    }
    PB_CUDA(b, cudaMemcpy(b->d_inst, hi.data(), sizeof(BatchInstance) * b->n, cudaMemcpyHostToDevice));
    return PEARL_OK;
}

int batch_launch(pearl_gpu_batch* b, const pearl_run_limits& L) {
    const NvtxRange range("pearl_gpu batch run");
    PB_CUDA(b, cudaSetDevice(b->device));
    PB_CUDA(b, cudaMemsetAsync(b->d_group_ctl, 0, sizeof(Ctl) * b->ngroups, b->stream));
    BatchArgs args{};
    args.inst = b->d_inst;
    args.order = b->d_order;
    args.first = b->d_first;
    args.block_group = b->d_block_group;
    args.group_block0 = b->d_group_block0;
    args.group_ctl = b->d_group_ctl;
    args.group_part = b->d_group_part;
    args.use_tma = b->use_tma ? 1 : 0;
    args.L = L;
    void* kargs[] = {&args};
    PB_CUDA(b, cudaEventRecord(b->ev0, b->stream));
    constexpr TileGeometry g = tile_geometry(8);
    // the mixed form's inner solve runs in a kernel of its own (all instances
    // of a batch share one precision, pearl_gpu_batch_set_precision)
    bool solve32 = false;
    for (auto* c : b->inst) solve32 = solve32 || c->P.mixed_cg;
    const void* kernel = solve32 ? (const void*)g8::pearl_batch_kernel_mixed : (const void*)g8::pearl_batch_kernel;
    PB_CUDA(b, cudaLaunchCooperativeKernel(kernel, dim3(b->grid), dim3(g.threads), kargs,
                                           b->use_tma ? g.tma_smem_bytes : 0, b->stream));
    b->launches++;
    PB_CUDA(b, cudaEventRecord(b->ev1, b->stream));
    PB_CUDA(b, cudaMemcpyAsync(b->h_ctls, b->d_ctls, sizeof(Ctl) * b->n, cudaMemcpyDeviceToHost, b->stream));
    PB_CUDA(b, cudaStreamSynchronize(b->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    for (int i = 0; i < b->n; ++i) *b->inst[i]->h_ctl = b->h_ctls[i];
    return PEARL_OK;
}

}  // namespace

extern "C" {

void pearl_gpu_batch_destroy(pearl_gpu_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto* c : b->inst) {
        if (c) c->d_ctl = nullptr;  // owned by the batch
        pearl_gpu_destroy(c);
    }
    cudaFree(b->d_ctls);
    if (b->h_ctls) cudaFreeHost(b->h_ctls);
    cudaFree(b->d_inst);
    cudaFree(b->d_order);
    cudaFree(b->d_first);
    cudaFree(b->d_block_group);
    cudaFree(b->d_group_block0);
    cudaFree(b->d_group_ctl);
    cudaFree(b->d_group_part);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
}

int pearl_gpu_batch_create(int n, const pearl_params* params, const int* nx, const int* ny, int device,
                           int group_blocks, pearl_gpu_batch** out) {
    if (!out || n < 1 || !params || !nx || !ny) return PEARL_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    pearl_gpu_batch* b = new pearl_gpu_batch();
    b->device = device;
    b->n = n;
    auto bail = [&](int rc) {
        pearl_gpu_batch_destroy(b);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(PEARL_ERR_NO_DEVICE);
    b->inst.assign(n, nullptr);
    if (cudaMalloc(&b->d_ctls, sizeof(Ctl) * n) != cudaSuccess ||
        cudaMallocHost(&b->h_ctls, sizeof(Ctl) * n) != cudaSuccess ||
        cudaMalloc(&b->d_inst, sizeof(BatchInstance) * n) != cudaSuccess)
        return bail(PEARL_ERR_CUDA);
    std::memset(b->h_ctls, 0, sizeof(Ctl) * n);
    bool tma = true;
    for (int i = 0; i < n; ++i) {
        const int rc = pearl_gpu_create(&params[i], nx[i], ny[i], device, &b->inst[i]);
        if (rc) return bail(rc);
        pearl_gpu_ctx* c = b->inst[i];
        set_geometry(c, 8);  // the batch kernel runs 256-thread blocks, two per SM
        cudaFree(c->d_ctl);  // the batch keeps every control block in one array
        c->d_ctl = b->d_ctls + i;
        c->B.ctl = c->d_ctl;
        if (cudaMemcpy(c->d_ctl, c->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(PEARL_ERR_CUDA);
        tma = tma && c->use_tma;
    }
    if (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
        return bail(PEARL_ERR_CUDA);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    const void* kernels[2] = {(const void*)g8::pearl_batch_kernel, (const void*)g8::pearl_batch_kernel_mixed};
    for (const void* k : kernels)
        if (tma && cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tile_geometry(8).tma_smem_bytes) != cudaSuccess)
            tma = false;
    b->per_sm = 1 << 30;
    for (const void* k : kernels) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, tile_geometry(8).threads,
                                                          tma ? tile_geometry(8).tma_smem_bytes : 0) != cudaSuccess ||
            n < 1)
            return bail(PEARL_ERR_CUDA);
        b->per_sm = std::min(b->per_sm, n);
    }
    b->tma_capable = tma;
    const int rc = batch_configure(b, group_blocks > 0 ? group_blocks : PEARL_BATCH_SIZED_GROUPS, tma, 0);
    if (rc) return bail(rc);
    *out = b;
    return PEARL_OK;
}

int pearl_gpu_batch_upload(pearl_gpu_batch* b, int i, const double* phi, const double* carbon, const double* mu,
                           const pearl_scalars* scalars) {
    if (!b || i < 0 || i >= b->n) return PEARL_ERR_INVALID_ARGUMENT;
    const int rc = pearl_gpu_upload(b->inst[i], phi, carbon, mu, scalars);
    if (rc) return bfail(b, rc, pearl_gpu_last_error(b->inst[i]));
    return PEARL_OK;
}

int pearl_gpu_batch_download(pearl_gpu_batch* b, int i, double* phi, double* carbon, double* mu,
                             pearl_scalars* scalars) {
    if (!b || i < 0 || i >= b->n) return PEARL_ERR_INVALID_ARGUMENT;
    const int rc = pearl_gpu_download(b->inst[i], phi, carbon, mu, scalars);
    if (rc) return bfail(b, rc, pearl_gpu_last_error(b->inst[i]));
    return PEARL_OK;
}

int pearl_gpu_batch_run(pearl_gpu_batch* b, const pearl_run_limits* limits, pearl_run_report* reports,
                        int* status) {
    if (!b || !limits || limits->max_steps < 1) return PEARL_ERR_INVALID_ARGUMENT;
    int rc = batch_launch(b, *limits);
    if (rc) return rc;
    int first_bad = PEARL_OK;
    for (int i = 0; i < b->n; ++i) {
        const Ctl& h = b->h_ctls[i];
        if (reports) {
            reports[i].steps = h.steps;
            reports[i].cg_total = h.cg_total;
            reports[i].cg_peak = h.cg_peak;
            reports[i].reached_stop = h.reached_stop;
            reports[i].last = h.last;
        }
        if (status) status[i] = h.status;
        if (h.status == PEARL_ERR_DEVICE_WAIT) first_bad = PEARL_ERR_DEVICE_WAIT;
    }
    if (first_bad) return bfail(b, first_bad, "device grid barrier wait exceeded its limit");
    return PEARL_OK;
}

int pearl_gpu_batch_autotune(pearl_gpu_batch* b, int steps, int* group_blocks, int* use_tma, int* tile_warps_x) {
    if (!b || steps < 1) return PEARL_ERR_INVALID_ARGUMENT;
    PB_CUDA(b, cudaSetDevice(b->device));
    // back up every instance's current state (5 planes) and control block
    std::vector<double*> backup(b->n, nullptr);
    auto release = [&]() {
        for (double* p : backup) cudaFree(p);
    };
    for (int i = 0; i < b->n; ++i) {
        pearl_gpu_ctx* c = b->inst[i];
        const size_t bytes = 5 * plane_elems(c) * sizeof(double);
        if (cudaMalloc(&backup[i], bytes) != cudaSuccess) {
            release();
            return bfail(b, PEARL_ERR_CUDA, "autotune backup allocation");
        }
        cudaMemcpyAsync(backup[i], c->B.phi[c->h_ctl->cur][0], bytes, cudaMemcpyDeviceToDevice, b->stream);
    }
    // the instances' host control blocks are authoritative (uploads update them)
    std::vector<Ctl> saved(b->n);
    for (int i = 0; i < b->n; ++i) saved[i] = *b->inst[i]->h_ctl;
    double best_ms = 1e300;
    int best_gb = b->group_blocks, best_wx = b->tile_wx;
    bool best_tma = b->use_tma;
    double best_o = b->pass_overhead_tiles;
    // equal groups of 1..16 blocks, and groups sized per instance with three
    // weights of a pass's fixed cost (in tiles of one block)
    struct Cand {
        int gb;
        double o;
    };
    const Cand cands[] = {{1, 0},  {2, 0},  {4, 0},  {8, 0},  {16, 0}, {PEARL_BATCH_SIZED_GROUPS, 1},
                          {PEARL_BATCH_SIZED_GROUPS, 4}, {PEARL_BATCH_SIZED_GROUPS, 16}};
    // one launch of `steps` steps per trial: the first steps of a run carry the
    // step-start energy and most rejected attempts, so single steps rank poorly
    pearl_run_limits L{steps, 0x7fffffffffffffffLL, 1e300, 1e300, 0};
    // tile shapes 32x16 (with and without TMA staging), 64x8 and 128x4
    struct Shape {
        int wx;
        bool tma;
    };
    std::vector<Shape> shapes;
    if (b->tma_capable) shapes.push_back({0, true});
    shapes.push_back({0, false});
    shapes.push_back({1, false});
    shapes.push_back({2, false});
    for (const Shape& sh : shapes) {
        const int tma = sh.tma ? 1 : 0;
        for (const Cand& cand : cands) {
            const int gb = cand.gb;
            if (gb > b->per_sm * b->sms) continue;
            if (gb == PEARL_BATCH_SIZED_GROUPS) b->pass_overhead_tiles = cand.o;
            int rc = batch_configure(b, gb, tma != 0, sh.wx);
            double ms = 0;
            if (rc == PEARL_OK) {
                rc = batch_launch(b, L);
                ms = b->last_ms;
            }
            // restore
            for (int i = 0; i < b->n; ++i) {
                pearl_gpu_ctx* c = b->inst[i];
                cudaMemcpyAsync(c->B.phi[saved[i].cur][0], backup[i], 5 * plane_elems(c) * sizeof(double),
                                cudaMemcpyDeviceToDevice, b->stream);
            }
            std::memcpy(b->h_ctls, saved.data(), sizeof(Ctl) * b->n);
            cudaMemcpyAsync(b->d_ctls, b->h_ctls, sizeof(Ctl) * b->n, cudaMemcpyHostToDevice, b->stream);
            cudaStreamSynchronize(b->stream);
            for (int i = 0; i < b->n; ++i) *b->inst[i]->h_ctl = saved[i];
            if (rc) {
                release();
                return rc;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best_gb = gb;
                best_tma = tma != 0;
                best_wx = sh.wx;
                if (gb == PEARL_BATCH_SIZED_GROUPS) best_o = cand.o;
            }
        }
    }
    release();
    b->pass_overhead_tiles = best_o;
    const int rc = batch_configure(b, best_gb, best_tma, best_wx);
    if (group_blocks) *group_blocks = best_gb;
    if (use_tma) *use_tma = best_tma ? 1 : 0;
    if (tile_warps_x) *tile_warps_x = 1 << best_wx;
    return rc;
}

int pearl_gpu_batch_plan(int n, const long long* tiles, int grid_blocks, int group_blocks, double pass_overhead_tiles,
                         int* group_of_instance, int* group_size, int* ngroups, double* longest) {
    if (n < 1 || !tiles || grid_blocks < 1 || !(pass_overhead_tiles >= 0) || !group_of_instance || !group_size ||
        !ngroups)
        return PEARL_ERR_INVALID_ARGUMENT;
    if (group_blocks != PEARL_BATCH_SIZED_GROUPS && (group_blocks < 1 || group_blocks > grid_blocks))
        return PEARL_ERR_INVALID_ARGUMENT;
    std::vector<long long> t(tiles, tiles + n);
    for (long long x : t)
        if (x < 1) return PEARL_ERR_INVALID_ARGUMENT;
    std::vector<int> sizes;
    std::vector<std::vector<int>> lists;
    const double m = plan_groups(t, grid_blocks, group_blocks, pass_overhead_tiles, sizes, lists);
    for (size_t g = 0; g < sizes.size(); ++g) {
        group_size[g] = sizes[g];
        for (int i : lists[g]) group_of_instance[i] = (int)g;
    }
    *ngroups = (int)sizes.size();
    if (longest) *longest = m;
    return PEARL_OK;
}

int pearl_gpu_batch_configure(pearl_gpu_batch* b, int group_blocks, int use_tma, int tile_warps_x) {
    if (!b) return PEARL_ERR_INVALID_ARGUMENT;
    const int wx = tile_warps_x == 1 ? 0 : tile_warps_x == 2 ? 1 : tile_warps_x == 4 ? 2 : tile_warps_x == 8 ? 3 : -1;
    if (wx < 0) return bfail(b, PEARL_ERR_INVALID_ARGUMENT, "tile_warps_x must be 1, 2, 4 or 8");
    PB_CUDA(b, cudaSetDevice(b->device));
    return batch_configure(b, group_blocks, use_tma != 0, wx);
}

int pearl_gpu_batch_set_precision(pearl_gpu_batch* b, int precision) {
    if (!b) return PEARL_ERR_INVALID_ARGUMENT;
    for (auto* c : b->inst) {
        const int rc = pearl_gpu_set_precision(c, precision);
        if (rc) return bfail(b, rc, "invalid precision");
    }
    return batch_configure(b, b->group_blocks, b->use_tma, b->tile_wx);
}

int pearl_gpu_batch_stats(const pearl_gpu_batch* b, long long* launches, int* grid_blocks, int* group_blocks,
                          double* last_kernel_ms) {
    if (!b) return PEARL_ERR_INVALID_ARGUMENT;
    if (launches) *launches = b->launches;
    if (grid_blocks) *grid_blocks = b->grid;
    if (group_blocks) *group_blocks = b->group_blocks;
    if (last_kernel_ms) *last_kernel_ms = b->last_ms;
    return PEARL_OK;
}

const char* pearl_gpu_batch_last_error(const pearl_gpu_batch* b) { return b ? b->error.c_str() : "null batch"; }

}  // extern "C"


// Uneven batches in one persistent launch, captured in a CUDA graph, and the
// autotuner that picks, per length, the radix order, elements per thread and
// tile shape of the SIMT tile kernels, and the stage arithmetic (FP32 SIMT or
// a split-precision tensor-core form) of ordinary plans in precision mode 3.
//
// An uneven batch is a list of groups (length n_i, count b_i) of 1D C2C
// transforms stored back to back.  Every group is planned with the ordinary
// planner; its launches become segments of one work list (segment, tile)
// executed by a single persistent kernel (batch_fft_kernel in fft_tile.cu),
// whose CTAs dequeue tiles from a global counter.  A segment that reads
// another segment's output (the next pass of a long transform, the second
// half of a Bluestein transform) waits for that segment's completion count.
// The counter reset and the launch are captured once into a CUDA graph and
// replayed while the buffers stay the same.
//
// The reference has no counterpart: it runs one plan per length, each as its
// own sequence of launches (core/fft/fft_api.cpp asdFftExecV2).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "../../include/asdsip_fft_ext.h"
#include "sipfft_internal.h"

namespace sipfft {

// ------------------------------------------------------------------------------------ tuner store
namespace {
std::mutex g_tune_mu;
std::map<int64_t, TuneChoice> g_tuned;
}  // namespace

bool tuned_choice(int64_t n, TuneChoice &out)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(n);
    if (it == g_tuned.end()) return false;
    out = it->second;
    return true;
}

void set_tuned_choice(int64_t n, const TuneChoice &c)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[n] = c;
}

namespace {

std::string gpu_name(int device)
{
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string s = prop.name;
    for (char &ch : s)
        if (ch == '"' || ch == '\n') ch = ' ';
    return s;
}

// Cache file: one JSON object per line,
// {"gpu": "...", "type": "c2c", "precision": "fp32", "n": 4096, "radices": [16,16,16], "maxe": 16,
//  "row_threads": 256, "us": 12.5, "plan_us": 30.1}
// radices / maxe / row_threads: the SIMT tile kernels' choice (us: its time);
// precision: the arithmetic that ran the whole plan fastest (plan_us).
bool parse_line(const std::string &line, std::string &gpu, int64_t &n, TuneChoice &c)
{
    auto field = [&](const char *key) -> std::string {
        const std::string k = std::string("\"") + key + "\":";
        size_t p = line.find(k);
        if (p == std::string::npos) return std::string();
        p += k.size();
        while (p < line.size() && line[p] == ' ') p++;
        size_t e = p;
        if (p < line.size() && line[p] == '"') {
            e = line.find('"', p + 1);
            return e == std::string::npos ? std::string() : line.substr(p + 1, e - p - 1);
        }
        if (p < line.size() && line[p] == '[') {
            e = line.find(']', p);
            return e == std::string::npos ? std::string() : line.substr(p + 1, e - p - 1);
        }
        while (e < line.size() && line[e] != ',' && line[e] != '}') e++;
        return line.substr(p, e - p);
    };
    gpu = field("gpu");
    const std::string ns = field("n"), rs = field("radices"), ms = field("maxe"), us = field("us");
    if (gpu.empty() || ns.empty() || line.find("\"radices\":") == std::string::npos || field("type") != "c2c")
        return false;
    n = std::atoll(ns.c_str());
    c.radices.clear();
    std::stringstream ss(rs);
    std::string tok;
    while (std::getline(ss, tok, ',')) c.radices.push_back(std::atoi(tok.c_str()));
    c.maxe = std::atoi(ms.c_str());
    c.us = std::atof(us.c_str());
    c.row_threads = std::atoi(field("row_threads").c_str());
    const std::string pr = field("precision");
    c.precision = pr == "fp16x3" ? 1 : (pr == "bf16x3" ? 2 : 0);
    c.plan_us = std::atof(field("plan_us").c_str());
    // empty radices: the planner's tile shape and radix order (only the arithmetic is recorded)
    return n > 0 && (c.radices.empty() || valid_radices(c.radices, n)) && c.row_threads >= 0 && c.row_threads <= 512;
}

}  // namespace

int load_tune_cache(const std::string &path, int device)
{
    std::ifstream f(path);
    if (!f) return 0;
    const std::string me = gpu_name(device);
    std::string line, gpu;
    int count = 0;
    while (std::getline(f, line)) {
        int64_t n = 0;
        TuneChoice c;
        if (parse_line(line, gpu, n, c) && gpu == me) {
            set_tuned_choice(n, c);
            count++;
        }
    }
    return count;
}

bool save_tune_cache(const std::string &path, int device)
{
    const std::string me = gpu_name(device);
    // keep other GPUs' entries, replace this GPU's
    std::vector<std::string> keep;
    {
        std::ifstream f(path);
        std::string line, gpu;
        while (std::getline(f, line)) {
            int64_t n = 0;
            TuneChoice c;
            if (parse_line(line, gpu, n, c) && gpu != me) keep.push_back(line);
        }
    }
    std::ofstream o(path, std::ios::trunc);
    if (!o) return false;
    for (const auto &l : keep) o << l << "\n";
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const auto &kv : g_tuned) {
        static const char *kForm[] = {"fp32", "fp16x3", "bf16x3"};
        const TuneChoice &c = kv.second;
        o << "{\"gpu\": \"" << me << "\", \"type\": \"c2c\", \"precision\": \"" << kForm[c.precision % 3]
          << "\", \"n\": " << kv.first << ", \"radices\": [";
        for (size_t i = 0; i < c.radices.size(); i++) o << (i ? "," : "") << c.radices[i];
        o << "], \"maxe\": " << c.maxe << ", \"row_threads\": " << c.row_threads << ", \"us\": " << c.us
          << ", \"plan_us\": " << c.plan_us << "}\n";
    }
    return static_cast<bool>(o);
}

// Candidate radix orders / elements per thread for one length.
std::vector<TuneChoice> tune_candidates(int64_t n)
{
    std::vector<TuneChoice> out;
    std::vector<int> base;
    if (!factor_radices(n, base)) return out;
    std::vector<std::vector<int>> orders;
    orders.push_back(base);
    std::vector<int> rev(base.rbegin(), base.rend());
    orders.push_back(rev);
    // powers of two split into radix-8 stages instead of 16
    {
        int64_t m = n;
        int twos = 0;
        while (m % 2 == 0) {
            m /= 2;
            twos++;
        }
        std::vector<int> r8;
        int t = twos;
        while (t >= 3) {
            r8.push_back(8);
            t -= 3;
        }
        if (t == 2) r8.push_back(4);
        if (t == 1) r8.push_back(2);
        std::vector<int> odd;
        if (factor_radices(m, odd)) {  // m is odd: only odd radices
            for (int x : odd) r8.push_back(x);
            orders.push_back(r8);
        }
        std::vector<int> oddfirst;
        for (int x : base)
            if (x % 2) oddfirst.push_back(x);
        for (int x : base)
            if (x % 2 == 0) oddfirst.push_back(x);
        orders.push_back(oddfirst);
    }
    std::sort(orders.begin(), orders.end());
    orders.erase(std::unique(orders.begin(), orders.end()), orders.end());
    for (const auto &o : orders) {
        for (int maxe : {8, 16}) {
            const int tpt = static_cast<int>((n + maxe - 1) / maxe);
            if (tpt > kBatchBlock) continue;
            // tile shape: transforms per tile so that a tile has about this many threads
            // (the batch kernel's CTA has 256)
            for (int threads : {128, 256}) {
                if (threads < tpt) continue;
                TuneChoice c;
                c.radices = o;
                c.maxe = maxe;
                c.row_threads = threads;
                out.push_back(c);
            }
        }
    }
    return out;
}

// ------------------------------------------------------------------------------------ batch plan
struct BatchPlan {
    int device = 0;
    bool forward = true;
    std::vector<int64_t> sizes, batches;
    std::vector<BatchSeg> segs;
    std::vector<int2> items;
    std::vector<std::string> seg_what;
    BatchSeg *d_segs = nullptr;
    int2 *d_items = nullptr;
    int *d_counters = nullptr;  // [0] = item counter, [1 + s] = tiles done of segment s
    size_t ws_bytes = 0;
    int grid = 1, block = kBatchBlock;
    bool compact = false;  // every segment's radices are <= kCompactMaxRadix (three CTAs per SM)
    size_t smem = 0;
    std::vector<TablePtr> tables;
    int64_t in_elems = 0, out_elems = 0;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *g_in = nullptr;
    void *g_out = nullptr;
    void *g_ws = nullptr;
    cudaStream_t g_stream = nullptr;
    std::mutex mu;
    ~BatchPlan()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        cudaFree(d_segs);
        cudaFree(d_items);
        cudaFree(d_counters);
        cudaGetLastError();
    }
};

namespace {

std::string build_batch_with(BatchPlan &bp)
{
    bp.segs.clear();
    bp.items.clear();
    bp.seg_what.clear();
    bp.tables.clear();
    bp.smem = 0;
    int64_t in_off = 0, ws_off = 0;
    struct Pending {
        int seg;
        int phase;
        double cost;
    };
    std::vector<Pending> order;
    for (size_t g = 0; g < bp.sizes.size(); g++) {
        const int64_t n = bp.sizes[g], b = bp.batches[g];
        if (n <= 0 || b <= 0) return "group with non-positive length or count";
        Plan p;
        p.fft_type = 0x10;
        p.direction = bp.forward ? 0x10 : 0x11;
        p.sizes = {n};
        p.strides = {1};
        p.batch = b;
        p.device = bp.device;
        p.use_tuned = true;
        // tiles of at most 256 threads x 16 points and a few tens of KB, so that
        // several CTAs of the one batch kernel share an SM: longer rows go multi-pass
        p.row_threads = 256;
        p.row_smem = 48 * 1024;
        p.max_row_n = kBatchMaxRowN;
        p.max_maxe = kBatchMaxe;
        p.max_radix = bp.compact ? kCompactMaxRadix : 16;
        std::string e = build_plan_1d(p);
        if (!e.empty()) return "length " + std::to_string(n) + ": " + e;
        const size_t ws0 = (p.ws_buf_bytes[0] + 255) / 256 * 256;
        const size_t ws1 = (p.ws_buf_bytes[1] + 255) / 256 * 256;
        for (size_t i = 0; i < p.steps.size(); i++) {
            const Step &s = p.steps[i];
            if (s.kind != StepKind::kTile) return "unsupported step kind in an uneven batch";
            BatchSeg sg{};
            sg.d = s.d;
            sg.d.in = nullptr;
            sg.d.out = nullptr;
            auto place = [&](Buf b, int &buf, int64_t &off) {
                switch (b) {
                    case Buf::kUserIn: buf = 0; off = in_off * 8; break;
                    case Buf::kUserOut: buf = 1; off = in_off * 8; break;
                    case Buf::kWs0: buf = 2; off = ws_off; break;
                    case Buf::kWs1: buf = 2; off = ws_off + static_cast<int64_t>(ws0); break;
                }
            };
            place(s.src, sg.in_buf, sg.in_off);
            place(s.dst, sg.out_buf, sg.out_off);
            sg.dep = i == 0 ? -1 : static_cast<int>(bp.segs.size()) - 1;
            sg.ntiles = static_cast<int>(s.d.num_tiles);
            sg.fwd = s.forward ? 1 : 0;
            if (s.d.tb * s.d.tpt > bp.block) return "tile shape exceeds the batch block size";
            if (s.maxe > kBatchMaxe) return "tile needs more points per thread than the batch kernel holds";
            // two buffers per CTA (the batch kernel prefetches its next item)
            bp.smem = std::max(bp.smem, 2 * static_cast<size_t>(s.d.tb) * s.d.pitch * sizeof(float2));
            const int phase = p.steps.size() == 1 ? 1 : (i == 0 ? 0 : static_cast<int>(i) + 1);
            order.push_back({static_cast<int>(bp.segs.size()), phase, double(s.d.n) * s.d.tb});
            bp.segs.push_back(sg);
            bp.seg_what.push_back(s.what);
        }
        for (auto &t : p.tables) bp.tables.push_back(t);
        in_off += n * b;
        ws_off += static_cast<int64_t>(ws0 + ws1);
    }
    bp.in_elems = bp.out_elems = in_off;
    bp.ws_bytes = static_cast<size_t>(ws_off);
    // producers before consumers; within a phase the heaviest tiles first
    std::stable_sort(order.begin(), order.end(), [](const Pending &a, const Pending &b) {
        if (a.phase != b.phase) return a.phase < b.phase;
        return a.cost > b.cost;
    });
    for (const Pending &pd : order)
        for (int t = 0; t < bp.segs[pd.seg].ntiles; t++) bp.items.push_back(make_int2(pd.seg, t));
    if (bp.items.size() > 0x7fffffff) return "too many tiles";
    const int per_sm = kernel_blocks_per_sm(batch_kernel_fn(bp.forward, bp.compact), bp.block, bp.smem);
    if (per_sm <= 0) return "batch kernel does not fit on an SM";
    bp.grid = per_sm * sm_count(bp.device);
    size_t bytes = bp.segs.size() * sizeof(BatchSeg);
    if (cudaMalloc(&bp.d_segs, bytes) != cudaSuccess ||
        cudaMemcpy(bp.d_segs, bp.segs.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&bp.d_items, bp.items.size() * sizeof(int2)) != cudaSuccess ||
        cudaMemcpy(bp.d_items, bp.items.data(), bp.items.size() * sizeof(int2), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMalloc(&bp.d_counters, (1 + bp.segs.size()) * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return "twiddle table: device allocation failed";
    }
    return std::string();
}

// The compact kernel (radices up to 10, three CTAs per SM) when every length
// factors into them (16 and 12 split), else the kernel with every radix.
std::string build_batch(BatchPlan &bp)
{
    bp.compact = true;
    std::string e = build_batch_with(bp);
    if (!e.empty() && e.find("needs a radix above") != std::string::npos) {
        bp.compact = false;
        e = build_batch_with(bp);
    }
    return e;
}

cudaError_t enqueue(BatchPlan &bp, const void *in, void *out, void *ws, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(bp.d_counters, 0, (1 + bp.segs.size()) * sizeof(int), st);
    if (e != cudaSuccess) return e;
    BatchBufs bufs{{const_cast<void *>(in), out, ws, nullptr}};
    return launch_batch(bp.grid, bp.block, bp.smem, bp.d_segs, bp.d_items, static_cast<int>(bp.items.size()),
                        bp.d_counters, bp.d_counters + 1, bufs, device_error_word(bp.device), bp.forward, bp.compact,
                        st);
}

std::mutex g_batch_mu;
std::map<void *, std::unique_ptr<BatchPlan>> g_batches;

BatchPlan *find_batch(void *h)
{
    std::lock_guard<std::mutex> lock(g_batch_mu);
    auto it = g_batches.find(h);
    return it == g_batches.end() ? nullptr : it->second.get();
}

}  // namespace

namespace {

// One uneven-batch launch over every group, timed (us per launch); false if it
// cannot be planned or run.
bool time_mix(const std::vector<int64_t> &sizes, const std::vector<int64_t> &rows_per, bool forward, int device,
              void *in, void *out, cudaEvent_t e0, cudaEvent_t e1, double &us)
{
    BatchPlan bp;
    bp.device = device;
    bp.forward = forward;
    bp.sizes = sizes;
    bp.batches = rows_per;
    if (!build_batch(bp).empty()) {
        cudaGetLastError();
        return false;
    }
    void *ws = nullptr;
    if (bp.ws_bytes && cudaMalloc(&ws, bp.ws_bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    bool ok = true;
    for (int rep = 0; rep < 2 && ok; rep++) ok = enqueue(bp, in, out, ws, 0) == cudaSuccess;
    cudaEventRecord(e0, 0);
    for (int rep = 0; rep < 4 && ok; rep++) ok = enqueue(bp, in, out, ws, 0) == cudaSuccess;
    cudaEventRecord(e1, 0);
    ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
    if (ws) cudaFree(ws);
    if (!ok) {
        cudaGetLastError();
        return false;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    us = ms * 1e3 / 4.0;
    return true;
}

// The per-length winners were timed one length at a time.  In the mixed
// launch every segment shares the grid and the CTA's shared memory is sized
// by the largest tile of any segment, so a winner's tile shape and radix
// order are kept only if the launch of all the groups together runs faster
// with them (lengths taken by decreasing bytes; the arithmetic choice of
// precision mode 3 is kept either way).
void accept_in_mix(const std::vector<int64_t> &sizes, const std::vector<int64_t> &rows_per,
                   const std::vector<int64_t> &targets, bool forward, int device, cudaEvent_t e0, cudaEvent_t e1)
{
    int64_t total = 0;
    for (size_t i = 0; i < sizes.size(); i++) total += sizes[i] * rows_per[i];
    void *in = nullptr, *out = nullptr;
    if (cudaMalloc(&in, total * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&out, total * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(in);
        return;  // no room for the whole mix: the per-length winners stand
    }
    cudaMemset(in, 0, total * sizeof(float2));
    // bytes of the launch whose tiles each tuned length shapes (as a group or as a pass)
    std::map<int64_t, int64_t> weight;
    for (size_t i = 0; i < sizes.size(); i++) {
        if (sizes[i] <= kBatchMaxRowN) weight[sizes[i]] += sizes[i] * rows_per[i];
        else
            for (int r : multipass_split(sizes[i])) weight[r] += sizes[i] * rows_per[i];
    }
    std::vector<std::pair<int64_t, int64_t>> order;  // (bytes, length)
    std::map<int64_t, TuneChoice> winners;
    for (const int64_t n : targets) {
        TuneChoice c;
        if (!tuned_choice(n, c) || c.radices.empty()) continue;
        winners[n] = c;
        order.push_back({weight[n], n});
        TuneChoice plain = c;  // the planner's defaults for the launch, the arithmetic kept
        plain.radices.clear();
        plain.maxe = 0;
        plain.row_threads = 0;
        set_tuned_choice(n, plain);
    }
    std::sort(order.rbegin(), order.rend());
    double best = 0.0;
    if (time_mix(sizes, rows_per, forward, device, in, out, e0, e1, best)) {
        for (const auto &o : order) {
            const TuneChoice keep = winners[o.second];
            TuneChoice plain = keep;
            plain.radices.clear();
            plain.maxe = 0;
            plain.row_threads = 0;
            set_tuned_choice(o.second, keep);
            double us = 0.0;
            if (time_mix(sizes, rows_per, forward, device, in, out, e0, e1, us) && us < best * 0.995)
                best = us;
            else
                set_tuned_choice(o.second, plain);
        }
    }
    cudaFree(in);
    cudaFree(out);
}

}  // namespace

// Times each candidate in the uneven-batch kernel (a one-group batch plan of
// about 4 M points of the length) and records the fastest; for lengths with a
// tensor-core stage also times the whole ordinary plan in each arithmetic.
// Returns the number of lengths tuned.
int autotune_lengths(const std::vector<int64_t> &sizes, const std::vector<int64_t> &rows_per, bool forward,
                     int device, std::string *err)
{
    int tuned = 0;
    int64_t max_elems = 0;
    for (size_t i = 0; i < sizes.size(); i++)
        max_elems = std::max(max_elems, std::max(sizes[i] * rows_per[i], int64_t(1) << 22) + sizes[i] * 16);
    if (max_elems == 0) return 0;
    float2 *buf = nullptr, *out = nullptr;
    if (cudaMalloc(&buf, max_elems * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&out, max_elems * sizeof(float2)) != cudaSuccess) {
        if (err) *err = "autotune: out of device memory";
        cudaGetLastError();
        cudaFree(buf);
        return 0;
    }
    cudaMemset(buf, 0, max_elems * sizeof(float2));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // The lengths whose tiles the uneven-batch kernel runs: groups of at most
    // 16384 points, and the pass lengths of the multi-pass split of longer rows
    // (their passes are column tiles of those lengths)
    std::vector<int64_t> targets;
    for (int64_t n : sizes) {
        if (n <= 16384) targets.push_back(n);
        if (n > kBatchMaxRowN)
            for (int r : multipass_split(n)) targets.push_back(r);
    }
    std::sort(targets.begin(), targets.end());
    targets.erase(std::unique(targets.begin(), targets.end()), targets.end());
    for (const int64_t n : targets) {
        TuneChoice best;
        best.us = 1e30;
        // enough transforms that a launch is not just its overhead
        const int64_t rows = std::max<int64_t>(16, std::min<int64_t>((int64_t(1) << 22) / n, 4096));
        for (TuneChoice c : tune_candidates(n)) {
            set_tuned_choice(n, c);
            // the uneven-batch kernel runs these tiles: time a one-group batch plan
            BatchPlan bp;
            bp.device = device;
            bp.forward = forward;
            bp.sizes = {n};
            bp.batches = {rows};
            if (!build_batch(bp).empty()) {
                cudaGetLastError();
                continue;
            }
            void *ws = nullptr;
            if (bp.ws_bytes && cudaMalloc(&ws, bp.ws_bytes) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            bool ok = true;
            for (int rep = 0; rep < 2 && ok; rep++) ok = enqueue(bp, buf, out, ws, 0) == cudaSuccess;
            cudaEventRecord(e0, 0);
            for (int rep = 0; rep < 5 && ok; rep++) ok = enqueue(bp, buf, out, ws, 0) == cudaSuccess;
            cudaEventRecord(e1, 0);
            ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
            if (ws) cudaFree(ws);
            if (!ok) {
                cudaGetLastError();
                continue;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            c.us = ms * 1e3 / 5.0;
            if (c.us < best.us) best = c;
        }
        // whole-plan arithmetic per length (ordinary plans in precision mode 3):
        // the FP32 kernels against the split-precision tensor-core forms
        TcConfig tcc;
        if (best.us < 1e29 && (tc_config(static_cast<int>(n), tcc) || tc_rows_config(static_cast<int>(n), tcc))) {
            best.plan_us = 1e30;
            for (int form = 0; form < 3; form++) {
                Plan q;
                q.fft_type = 0x10;
                q.direction = forward ? 0x10 : 0x11;
                q.sizes = {n};
                q.batch = rows;
                q.device = device;
                q.precision = form;
                if (!build_plan_1d(q).empty() || q.ws_bytes > 0) continue;
                bool ok = true;
                for (int rep = 0; rep < 2 && ok; rep++) ok = execute_plan(q, buf, out, 0) == cudaSuccess;
                cudaEventRecord(e0, 0);
                for (int rep = 0; rep < 5 && ok; rep++) ok = execute_plan(q, buf, out, 0) == cudaSuccess;
                cudaEventRecord(e1, 0);
                if (!ok || cudaEventSynchronize(e1) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                const double us = ms * 1e3 / 5.0;
                if (us < best.plan_us) {
                    best.plan_us = us;
                    best.precision = form;
                }
            }
            if (best.plan_us >= 1e29) best.plan_us = 0.0;
        }
        if (best.us < 1e29) {
            set_tuned_choice(n, best);
            tuned++;
        }
    }
    cudaFree(buf);
    cudaFree(out);
    accept_in_mix(sizes, rows_per, targets, forward, device, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return tuned;
}

}  // namespace sipfft

using sipfft::BatchPlan;

extern "C" {

int32_t asdFftBatchPlanCreate(void **plan, const int64_t *sizes, const int64_t *batches, int32_t ngroups,
                              int32_t direction, const char *tune_cache)
{
    if (!plan || !sizes || !batches || ngroups <= 0) return AsdSip::ACL_ERROR_INVALID_PARAM;
    if (direction != AsdSip::ASCEND_FFT_FORWARD && direction != AsdSip::ASCEND_FFT_INVERSE)
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    try {
        auto bp = std::make_unique<BatchPlan>();
        if (cudaGetDevice(&bp->device) != cudaSuccess || sipfft::configure_kernels(bp->device) != cudaSuccess) {
            cudaGetLastError();
            return AsdSip::ACL_ERROR_INTERNAL_ERROR;
        }
        bp->forward = direction == AsdSip::ASCEND_FFT_FORWARD;
        bp->sizes.assign(sizes, sizes + ngroups);
        bp->batches.assign(batches, batches + ngroups);
        for (int i = 0; i < ngroups; i++)
            if (sizes[i] <= 0 || sizes[i] > (int64_t(1) << 27) || batches[i] <= 0)
                return AsdSip::ACL_ERROR_INVALID_PARAM;
        if (tune_cache && *tune_cache) sipfft::load_tune_cache(tune_cache, bp->device);
        std::string e = sipfft::build_batch(*bp);
        if (!e.empty()) {
            sipfft::set_last_error("asdFftBatchPlanCreate: " + e);
            if (std::getenv("ASDSIP_FFT_LOG")) std::fprintf(stderr, "[asdsip_fft] batch plan: %s\n", e.c_str());
            return e.rfind("twiddle table", 0) == 0 ? AsdSip::ACL_ERROR_INTERNAL_ERROR
                                                    : AsdSip::ACL_ERROR_API_NOT_SUPPORT;
        }
        void *h = bp.get();
        std::lock_guard<std::mutex> lock(sipfft::g_batch_mu);
        sipfft::g_batches.emplace(h, std::move(bp));
        *plan = h;
        return AsdSip::ACL_SUCCESS;
    } catch (...) {
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
}

int32_t asdFftBatchGetWorkspaceSize(void *plan, size_t *bytes)
{
    BatchPlan *bp = sipfft::find_batch(plan);
    if (!bp || !bytes) return AsdSip::ACL_ERROR_INVALID_PARAM;
    *bytes = bp->ws_bytes;
    return AsdSip::ACL_SUCCESS;
}

int32_t asdFftBatchExec(void *plan, const void *input, void *output, void *workspace, void *stream, int32_t use_graph)
{
    BatchPlan *bp = sipfft::find_batch(plan);
    if (!bp) return AsdSip::ACL_ERROR_INVALID_PARAM;
    if (!input || !output || input == output) return AsdSip::ACL_ERROR_INVALID_PARAM;
    if (bp->ws_bytes > 0 && !workspace) return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    if ((reinterpret_cast<uintptr_t>(input) & 7) || (reinterpret_cast<uintptr_t>(output) & 7))
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(bp->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (!use_graph) {
        e = sipfft::enqueue(*bp, input, output, workspace, st);
    } else {
        if (!bp->gexec || bp->g_in != input || bp->g_out != output || bp->g_ws != workspace || bp->g_stream != st) {
            if (bp->gexec) cudaGraphExecDestroy(bp->gexec);
            if (bp->graph) cudaGraphDestroy(bp->graph);
            bp->gexec = nullptr;
            bp->graph = nullptr;
            cudaStream_t cap = st;
            bool own = false;
            if (cap == nullptr) {  // the legacy default stream cannot be captured
                if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
                    cudaGetLastError();
                    return AsdSip::ACL_ERROR_INTERNAL_ERROR;
                }
                own = true;
            }
            e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t e2 = sipfft::enqueue(*bp, input, output, workspace, cap);
                e = cudaStreamEndCapture(cap, &bp->graph);
                if (e == cudaSuccess) e = e2;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&bp->gexec, bp->graph, 0);
            if (own) cudaStreamDestroy(cap);
            if (e != cudaSuccess) {
                sipfft::set_last_error(std::string("asdFftBatchExec: graph capture: ") + cudaGetErrorString(e));
                cudaGetLastError();
                return AsdSip::ACL_ERROR_INTERNAL_ERROR;
            }
            bp->g_in = input;
            bp->g_out = output;
            bp->g_ws = workspace;
            bp->g_stream = st;
        }
        e = cudaGraphLaunch(bp->gexec, st);
    }
    if (e != cudaSuccess) {
        sipfft::set_last_error(std::string("asdFftBatchExec: ") + cudaGetErrorString(e));
        cudaGetLastError();
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    return AsdSip::ACL_SUCCESS;
}

int32_t asdFftBatchPlanDestroy(void *plan)
{
    std::unique_ptr<BatchPlan> victim;
    {
        std::lock_guard<std::mutex> lock(sipfft::g_batch_mu);
        auto it = sipfft::g_batches.find(plan);
        if (it == sipfft::g_batches.end()) return AsdSip::ACL_ERROR_INVALID_PARAM;
        victim = std::move(it->second);
        sipfft::g_batches.erase(it);
    }
    std::lock_guard<std::mutex> lock(victim->mu);
    return AsdSip::ACL_SUCCESS;
}

int64_t asdFftBatchDescribe(void *plan, char *buf, int64_t len)
{
    BatchPlan *bp = sipfft::find_batch(plan);
    if (!bp) return -1;
    std::ostringstream o;
    o << "groups=" << bp->sizes.size() << " segments=" << bp->segs.size() << " items=" << bp->items.size()
      << " grid=" << bp->grid << " block=" << bp->block << " smem=" << bp->smem << " workspace=" << bp->ws_bytes
      << " kernel=" << (bp->compact ? "compact radices <= 10" : "every radix") << "\n";
    for (size_t i = 0; i < bp->segs.size(); i++) {
        const auto &s = bp->segs[i];
        o << "  seg " << i << " n=" << s.d.n << " tiles=" << s.ntiles << " tb=" << s.d.tb << " tpt=" << s.d.tpt
          << " radices=";
        for (int k = 0; k < s.d.nstages; k++) o << (k ? "x" : "") << s.d.radix[k];
        o << " dep=" << s.dep << " " << bp->seg_what[i] << "\n";
    }
    const std::string str = o.str();
    if (buf && len > 0) {
        const int64_t n = std::min<int64_t>(len - 1, static_cast<int64_t>(str.size()));
        std::memcpy(buf, str.data(), static_cast<size_t>(n));
        buf[n] = '\0';
    }
    return static_cast<int64_t>(str.size()) + 1;
}

int32_t asdFftAutotune(const int64_t *sizes, const int64_t *rows, int32_t n, int32_t direction,
                       const char *cache_path)
{
    if (!sizes || !rows || n <= 0) return AsdSip::ACL_ERROR_INVALID_PARAM;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || sipfft::configure_kernels(dev) != cudaSuccess) {
        cudaGetLastError();
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    std::vector<int64_t> s(sizes, sizes + n), r(rows, rows + n);
    for (auto &x : r) x = std::max<int64_t>(1, std::min<int64_t>(x, 256));
    std::string err;
    sipfft::autotune_lengths(s, r, direction == AsdSip::ASCEND_FFT_FORWARD, dev, &err);
    if (!err.empty()) return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    if (cache_path && *cache_path && !sipfft::save_tune_cache(cache_path, dev)) return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    return AsdSip::ACL_SUCCESS;
}

int32_t asdFftTuneCacheLoad(const char *cache_path)
{
    int dev = 0;
    if (!cache_path || cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return sipfft::load_tune_cache(cache_path, dev);
}

}  // extern "C"

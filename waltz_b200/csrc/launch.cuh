// Host side of the stage launches: a Sink either launches each stage at once
// on a stream (one field per call) or records it for a batched launch (many
// fields per call). A recorded batch is replayed stage by stage: all fields'
// k-th stage of one pipeline phase and of one op type become one launch of
// op_batch_kernel over a device table of their parameters.
#pragma once
#include "ops.cuh"

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <vector>

namespace wb {

// Dynamic shared memory above 48 KiB needs a per-kernel opt-in, per device.
template <class K> static void opt_in_smem(K kernel, size_t bytes, int& device, size_t& granted) {
    if (bytes <= 48 * 1024 && device != -1) return;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != device) granted = 0;
    if (bytes > granted || dev != device) {
        const size_t want = std::max<size_t>(bytes, 48 * 1024);
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(want)),
              "kernel shared memory");
        granted = want;
        device = dev;
    }
}

template <class Op> static void launch_op(const typename Op::Params& p, uint32_t blocks, size_t smem, cudaStream_t s) {
    if (!blocks) return;
    static thread_local int device = -1;
    static thread_local size_t granted = 0;
    constexpr auto kernel = op_kernel_for<Op>();
    opt_in_smem(kernel, smem, device, granted);
    kernel<<<blocks, Op::kThreads, smem, s>>>(p);
    note_launch();
    check(cudaGetLastError(), "kernel launch");
}

template <class Op>
static void launch_op_batch(const void* table, const uint32_t* starts, uint32_t count, uint32_t blocks, size_t smem,
                            cudaStream_t s) {
    if (!blocks) return;
    static thread_local int device = -1;
    static thread_local size_t granted = 0;
    opt_in_smem(op_batch_kernel<Op>, smem, device, granted);
    op_batch_kernel<Op><<<blocks, Op::kThreads, smem, s>>>(static_cast<const typename Op::Params*>(table), starts,
                                                           count);
    note_launch();
    check(cudaGetLastError(), "batched kernel launch");
}

// Resident CTAs of a kernel on this device (occupancy at its block size and
// shared memory, times the SM count).
template <class K> static uint32_t resident_ctas(K kernel, int threads, size_t smem) {
    int dev = 0, sms = 0, occ = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem), "occupancy");
    return uint32_t(std::max(sms, 1) * std::max(occ, 1));
}

template <class Op>
static void launch_op_queue(const void* table, const uint32_t* starts, uint32_t count, uint32_t blocks, size_t smem,
                            uint32_t* ticket, uint32_t share, cudaStream_t s) {
    if (!blocks) return;
    static thread_local int device = -1;
    static thread_local size_t granted = 0;
    opt_in_smem(op_queue_kernel<Op>, smem, device, granted);
    // one share of the resident CTAs: the parallel branches of the batch
    // graph each keep their queues on their share of the GPU
    const uint32_t slots = resident_ctas(op_queue_kernel<Op>, Op::kThreads, smem);
    const uint32_t grid = std::min(blocks, std::max(1u, (slots + share - 1) / share));
    op_queue_kernel<Op><<<grid, Op::kThreads, smem, s>>>(static_cast<const typename Op::Params*>(table), starts,
                                                         count, ticket);
    note_launch();
    check(cudaGetLastError(), "queued kernel launch");
}

// One recorded stage of one field.
struct OpRecord {
    virtual ~OpRecord() = default;
    virtual const void* kind() const = 0;
    virtual uint32_t blocks() const = 0;
    virtual size_t smem() const = 0;
    virtual size_t param_size() const = 0;
    virtual size_t param_align() const = 0;
    virtual void write_params(void* dst) const = 0;
    // a whole group of records of this kind: one batched launch (or, for
    // records that cannot be batched, one launch each)
    virtual void launch_group(const std::vector<const OpRecord*>& group, const void* table, const uint32_t* starts,
                              uint32_t blocks, size_t smem, cudaStream_t s) const = 0;
    // the same group as a persistent work queue (ticket zeroed beforehand)
    virtual void launch_queue(const std::vector<const OpRecord*>& group, const void* table, const uint32_t* starts,
                              uint32_t blocks, size_t smem, uint32_t* ticket, uint32_t share, cudaStream_t s) const {
        (void)ticket;
        (void)share;
        launch_group(group, table, starts, blocks, smem, s);
    }
};

template <class Op> struct OpRec final : OpRecord {
    typename Op::Params p;
    uint32_t nb;
    size_t sm;
    OpRec(const typename Op::Params& params, uint32_t b, size_t s) : p(params), nb(b), sm(s) {}
    static const void* tag() {
        static const char t = 0;
        return &t;
    }
    const void* kind() const override { return tag(); }
    uint32_t blocks() const override { return nb; }
    size_t smem() const override { return sm; }
    size_t param_size() const override { return sizeof(p); }
    size_t param_align() const override { return alignof(typename Op::Params); }
    void write_params(void* dst) const override { std::memcpy(dst, &p, sizeof(p)); }
    void launch_group(const std::vector<const OpRecord*>& group, const void* table, const uint32_t* starts,
                      uint32_t blocks, size_t smem, cudaStream_t s) const override {
        launch_op_batch<Op>(table, starts, uint32_t(group.size()), blocks, smem, s);
    }
    void launch_queue(const std::vector<const OpRecord*>& group, const void* table, const uint32_t* starts,
                      uint32_t blocks, size_t smem, uint32_t* ticket, uint32_t share, cudaStream_t s) const override {
        launch_op_queue<Op>(table, starts, uint32_t(group.size()), blocks, smem, ticket, share, s);
    }
};

// A stage without a batched form (the tensor-core matrix transform): each
// field's launch is kept as is.
struct DirectRec final : OpRecord {
    std::function<void(cudaStream_t)> fn;
    explicit DirectRec(std::function<void(cudaStream_t)> f) : fn(std::move(f)) {}
    static const void* tag() {
        static const char t = 0;
        return &t;
    }
    const void* kind() const override { return tag(); }
    uint32_t blocks() const override { return 0; }
    size_t smem() const override { return 0; }
    size_t param_size() const override { return 0; }
    size_t param_align() const override { return 1; }
    void write_params(void*) const override {}
    void launch_group(const std::vector<const OpRecord*>& group, const void*, const uint32_t*, uint32_t, size_t,
                      cudaStream_t s) const override {
        for (const OpRecord* r : group) static_cast<const DirectRec*>(r)->fn(s);
    }
};

// Pipeline phases, in order; a field's stages keep their order inside one.
enum Phase : int {
    PH_INIT = 0, PH_FORWARD, PH_QUANT, PH_ENCODE, PH_DIRECTORY, PH_INVERSE, PH_SIDE,
    PH_DCHECK, PH_DECODE, PH_QPATCH, PH_DINVERSE, PH_RPATCH,
};

struct Recorder {
    struct Entry {
        int phase, index;
        std::unique_ptr<OpRecord> rec;
    };
    std::vector<Entry> entries;
    int phase = 0, index = 0;
    void begin_field() { phase = 0, index = 0; }
    void set_phase(int p) {
        if (p != phase) index = 0;
        phase = p;
    }
    void add(std::unique_ptr<OpRecord> r) { entries.push_back({phase, index++, std::move(r)}); }
};

struct Sink {
    cudaStream_t stream = nullptr;
    Recorder* rec = nullptr;
    bool many = false; // many fields share the GPU: prefer fewer, larger blocks of work per field
    template <class Op> void run(const typename Op::Params& p, uint32_t blocks, size_t smem = 0) {
        if (rec) rec->add(std::make_unique<OpRec<Op>>(p, blocks, smem));
        else launch_op<Op>(p, blocks, smem, stream);
    }
    void zero(void* ptr, size_t bytes) {
        if (!bytes) return;
        if (rec) {
            const uint64_t vec = bytes / 16 + 1;
            run<ZeroOp>(ZeroOp::Params{ptr, bytes}, uint32_t(std::min<uint64_t>((vec + 255) / 256, 1024)));
        } else {
            check(cudaMemsetAsync(ptr, 0, bytes, stream), "memset");
        }
    }
    void direct(std::function<void(cudaStream_t)> fn) {
        if (rec) rec->add(std::make_unique<DirectRec>(std::move(fn)));
        else fn(stream);
    }
    void phase(int p) {
        if (rec) rec->set_phase(p);
    }
    void mark(const char* name) {
        if (!rec) stage_clock().mark(name, stream);
    }
};

// A recorded batch laid out for replay: steps in (phase, index) order, each a
// list of groups of one kind, and one device table with every group's
// parameters and block starts.
struct BatchPlan {
    struct Group {
        std::vector<const OpRecord*> recs;
        size_t table_off = 0, starts_off = 0;
        uint32_t blocks = 0;
        size_t smem = 0;
        uint32_t ticket = 0; // work-queue form: index of its ticket word
    };
    std::vector<std::vector<Group>> steps;
    std::vector<unsigned char> host; // the table image
    size_t tickets_off = 0;          // work-queue tickets, one u32 per group
    uint32_t tickets = 0;
    size_t bytes() const { return host.size(); }

    static BatchPlan make(const Recorder& r) {
        BatchPlan plan;
        std::map<std::pair<int, int>, std::vector<const OpRecord*>> slots;
        for (const auto& e : r.entries) slots[{e.phase, e.index}].push_back(e.rec.get());
        size_t at = 0;
        auto place = [&](size_t bytes, size_t align) {
            at = (at + align - 1) / align * align;
            const size_t off = at;
            at += bytes;
            return off;
        };
        for (auto& [slot, recs] : slots) {
            std::vector<Group> groups;
            std::map<const void*, size_t> index;
            for (const OpRecord* rec : recs) {
                auto it = index.find(rec->kind());
                if (it == index.end()) {
                    it = index.emplace(rec->kind(), groups.size()).first;
                    groups.emplace_back();
                }
                groups[it->second].recs.push_back(rec);
            }
            for (Group& g : groups) {
                const OpRecord* first = g.recs.front();
                const size_t stride = first->param_size(); // the kernel indexes a C array of Params
                g.table_off = place(stride * g.recs.size(), std::max<size_t>(first->param_align(), 64));
                g.starts_off = place(4 * (g.recs.size() + 1), 16);
                for (const OpRecord* rec : g.recs) {
                    g.smem = std::max(g.smem, rec->smem());
                    g.blocks += rec->blocks();
                }
            }
            for (Group& g : groups) g.ticket = plan.tickets++;
            plan.steps.push_back(std::move(groups));
        }
        plan.tickets_off = place(4 * size_t(plan.tickets + 1), 256);
        plan.host.assign(at, 0);
        for (auto& groups : plan.steps)
            for (Group& g : groups) {
                const size_t stride = g.recs.front()->param_size();
                uint32_t* starts = reinterpret_cast<uint32_t*>(plan.host.data() + g.starts_off);
                uint32_t b = 0;
                for (size_t k = 0; k < g.recs.size(); ++k) {
                    g.recs[k]->write_params(plan.host.data() + g.table_off + k * stride);
                    starts[k] = b;
                    b += g.recs[k]->blocks();
                }
                starts[g.recs.size()] = b;
            }
        return plan;
    }

    // Launches every step on `s`, reading the parameters from `table` (the
    // device copy of `host`); `queue`: each step as a persistent work queue
    // on 1/`share` of the resident CTAs (`share` plans run side by side),
    // its tickets zeroed first (a memset node of the captured graph).
    void execute(unsigned char* table, cudaStream_t s, bool queue = false, uint32_t share = 1) const {
        uint32_t* tick = reinterpret_cast<uint32_t*>(table + tickets_off);
        if (queue) check(cudaMemsetAsync(tick, 0, 4 * size_t(tickets), s), "ticket reset");
        for (const auto& groups : steps)
            for (const Group& g : groups) {
                const uint32_t* starts = reinterpret_cast<const uint32_t*>(table + g.starts_off);
                if (queue) g.recs.front()->launch_queue(g.recs, table + g.table_off, starts, g.blocks, g.smem,
                                                        tick + g.ticket, share, s);
                else g.recs.front()->launch_group(g.recs, table + g.table_off, starts, g.blocks, g.smem, s);
            }
    }
};

} // namespace wb

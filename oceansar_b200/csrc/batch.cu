// Scene batch engine (see batch.cuh): slot table management and the launch sequence of
// one step.  No counterpart in the reference, whose sar_raw (sar_raw_nompi.py:32-641)
// simulates one scene per call; a slot runs that per-pulse body for its scene.
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "batch.cuh"

namespace ocs {

__global__ void batch_advance_kernel(const __grid_constant__ BatchRef b) {
    for (int s = threadIdx.x; s < b.nslots; s += blockDim.x)
        if (slot_live(b.slots[s])) b.slots[s].counter += 1;
}

struct HostSlot {
    bool used = false;
    int rows_key = -1, cols_key = -1, prog = 0, nout = 0;
    int kind = kSlotStd;                          // pulse-kernel class
    bool choppy = false;                          // runs the choppy step after the column pass
    long long rows_items = 0, cols_items = 0;     // work items of the row / column pass
    long long pulse_items[5] = {0, 0, 0, 0, 0};   // pulse-kernel items per width class
    long long rows_smem = 0, cols_smem = 0;
};

}  // namespace ocs

using namespace ocs;

// Slot writes go through pinned staging (one region per slot) so that they are ordered on
// the caller's stream without blocking the host; a slot's region is reused only after the
// event of its previous copies has completed.
struct ocs_batch {
    int max_slots = 0;
    int precision = 0;
    SlotState *d_slots = nullptr;
    char *d_sargs = nullptr;
    char *d_pargs = nullptr;
    char *d_cargs = nullptr;              // choppy-step arguments of choppy scenes
    char *h_stage = nullptr;              // pinned: [max_slots][stage_bytes]
    size_t sbytes = 0, pbytes = 0, cbytes = 0, stage_bytes = 0;
    std::vector<cudaEvent_t> staged;      // per slot: its last staging copies
    std::vector<HostSlot> host;
};

static void batch_free(ocs_batch *b) {
    for (cudaEvent_t e : b->staged)
        if (e) cudaEventDestroy(e);
    cudaFree(b->d_slots);
    cudaFree(b->d_sargs);
    cudaFree(b->d_pargs);
    cudaFree(b->d_cargs);
    cudaFreeHost(b->h_stage);
    delete b;
}

extern "C" int ocs_batch_create(int32_t max_slots, int32_t precision, ocs_batch **out) {
    if (!out || max_slots < 1 || max_slots > kMaxSlots) return OCS_ERR_ARG;
    if (precision != OCS_PREC_F64 && precision != OCS_PREC_MIXED) return OCS_ERR_ARG;
    *out = nullptr;
    ocs_batch *b = new ocs_batch;
    b->max_slots = max_slots;
    b->precision = precision;
    b->sbytes = (surface_args_bytes() + 255) & ~(size_t)255;
    b->pbytes = (pulse_args_bytes() + 255) & ~(size_t)255;
    b->cbytes = (choppy_args_bytes() + 255) & ~(size_t)255;
    b->stage_bytes = ((sizeof(SlotState) + 255) & ~(size_t)255) + b->sbytes + b->pbytes + b->cbytes;
    b->host.resize(max_slots);
    b->staged.assign(max_slots, nullptr);
    cudaError_t e = cudaMalloc(&b->d_slots, sizeof(SlotState) * max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_sargs, b->sbytes * max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_pargs, b->pbytes * max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_cargs, b->cbytes * max_slots);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_stage, b->stage_bytes * max_slots);
    for (int i = 0; i < max_slots && e == cudaSuccess; ++i)
        e = cudaEventCreateWithFlags(&b->staged[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMemset(b->d_slots, 0, sizeof(SlotState) * max_slots);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        batch_free(b);
        return OCS_ERR_CUDA;
    }
    *out = b;
    return OCS_OK;
}

extern "C" int ocs_batch_destroy(ocs_batch *b) {
    if (!b) return OCS_ERR_ARG;
    const cudaError_t e = cudaDeviceSynchronize();
    batch_free(b);
    return e == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

extern "C" int ocs_batch_set(ocs_batch *b, int32_t slot, const ocs_scene_desc *sc, void *stream) {
    if (!b || !sc || slot < 0 || slot >= b->max_slots || !sc->surface || !sc->pulse) return OCS_ERR_ARG;
    const ocs_surface_desc *sd = sc->surface;
    const ocs_pulse_desc *pd = sc->pulse;
    if (!sc->t_d || !sc->add_d || !sc->az_now_d || !sc->flags_d || !sc->tmod_d) return OCS_ERR_ARG;
    if (sd->nx != pd->nx || sd->ny != pd->ny) return OCS_ERR_ARG;
    const int tile_rows = sc->tile_rows == 0 ? 64 : sc->tile_rows;
    if (tile_rows < 1 || tile_rows > 128) return OCS_ERR_ARG;
    HostSlot h;
    h.kind = pulse_kind(pd);
    if (b->precision == OCS_PREC_MIXED && h.kind == kSlotStd && !pulse_split_ok(pd)) return OCS_ERR_UNSUPPORTED;
    h.rows_key = surface_key(sd->nx);
    h.cols_key = surface_key(sd->ny);
    if (h.rows_key < 0 || h.cols_key < 0) return OCS_ERR_UNSUPPORTED;
    h.rows_smem = surface_rows_smem(h.rows_key, sd->nx);
    h.cols_smem = surface_cols_smem(h.cols_key, sd->ny);
    if (h.rows_smem < 0 || h.cols_smem < 0) return OCS_ERR_SIZE;
    h.nout = pd->npol * pd->nch;
    h.rows_items = sd->ny / 2 + 1;
    {
        const int tile = surface_cols_tile(h.cols_key);
        h.cols_items = (long long)((sd->nfields + 1) / 2) * ((sd->nx + tile - 1) / tile);
    }
    for (int w : {1, 2, 4})
        h.pulse_items[w] = batch_pulse_items(sd->nx, sd->ny, tile_rows, h.nout, b->precision, w);
    h.used = true;

    // the slot's staging region is free once its previous copies have run
    if (cudaEventSynchronize(b->staged[slot]) != cudaSuccess) return OCS_ERR_CUDA;
    char *stage = b->h_stage + b->stage_bytes * slot;
    char *st_slot = stage;
    char *st_sargs = stage + ((sizeof(SlotState) + 255) & ~(size_t)255);
    char *st_pargs = st_sargs + b->sbytes;
    char *st_cargs = st_pargs + b->pbytes;
    memset(stage, 0, b->stage_bytes);
    int st = surface_args_fill(sd, st_sargs, &h.prog);
    if (st != OCS_OK) return st;
    st = pulse_args_fill(pd, st_pargs);
    if (st != OCS_OK) return st;
    if (sc->choppy) {
        if (sc->choppy->n != (int64_t)sd->nx * sd->ny) return OCS_ERR_ARG;
        st = choppy_args_fill(sc->choppy, st_cargs);
        if (st != OCS_OK) return st;
        h.choppy = true;
    }

    SlotState s;
    memset(&s, 0, sizeof(s));
    s.active = 1;
    s.counter = 0;
    s.az_steps = pd->az_steps;
    s.nx = sd->nx;
    s.ny = sd->ny;
    s.rows_key = h.rows_key;
    s.cols_key = h.cols_key;
    s.npair = (sd->nfields + 1) / 2;
    s.nfields = sd->nfields;
    s.nout = h.nout;
    s.tile_rows = tile_rows;
    s.prog = h.prog;
    s.kind = h.kind;
    s.t_tab = sc->t_d;
    s.add_tab = sc->add_d;
    s.swrot_tab = reinterpret_cast<const float2 *>(sc->swell_rot_d);
    s.aznow_tab = sc->az_now_d;
    s.flags_tab = sc->flags_d;
    s.tmod_tab = sc->tmod_d;
    s.sargs = b->d_sargs + b->sbytes * slot;
    s.pargs = b->d_pargs + b->pbytes * slot;
    s.cargs = h.choppy ? b->d_cargs + b->cbytes * slot : nullptr;
    memcpy(st_slot, &s, sizeof(s));
    cudaStream_t cs = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(b->d_sargs + b->sbytes * slot, st_sargs, b->sbytes, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_pargs + b->pbytes * slot, st_pargs, b->pbytes, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess && h.choppy)
        e = cudaMemcpyAsync(b->d_cargs + b->cbytes * slot, st_cargs, b->cbytes, cudaMemcpyHostToDevice, cs);
    // the slot record last: kernels that run after it see complete arguments
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_slots + slot, st_slot, sizeof(s), cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaEventRecord(b->staged[slot], cs);
    if (e != cudaSuccess) return OCS_ERR_CUDA;
    b->host[slot] = h;
    return OCS_OK;
}

extern "C" int ocs_batch_clear(ocs_batch *b, int32_t slot, void *stream) {
    if (!b || slot < 0 || slot >= b->max_slots) return OCS_ERR_ARG;
    if (cudaEventSynchronize(b->staged[slot]) != cudaSuccess) return OCS_ERR_CUDA;
    int *zero = reinterpret_cast<int *>(b->h_stage + b->stage_bytes * slot);
    *zero = 0;
    cudaStream_t cs = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(&b->d_slots[slot].active, zero, sizeof(int), cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaEventRecord(b->staged[slot], cs);
    if (e != cudaSuccess) return OCS_ERR_CUDA;
    b->host[slot] = HostSlot();
    return OCS_OK;
}

// Launch classes of the slots in use: row / column transform lengths (with the largest
// shared memory each needs) and pulse-kernel (class, width) pairs.
struct ClassLaunch {
    long long smem = 0;     // largest shared memory of the class's slots
    long long items = 0;    // items of all the class's slots (the grid)
};

struct BatchPlan {
    std::vector<std::pair<std::pair<int, int>, ClassLaunch>> rows;   // (length, program)
    std::vector<std::pair<int, ClassLaunch>> cols;
    std::vector<std::pair<std::pair<int, int>, long long>> widths;    // ((kind, width class), items)
    bool choppy = false;                                              // some slot runs the choppy step
};

static BatchPlan batch_plan(const ocs_batch *b) {
    std::map<std::pair<int, int>, ClassLaunch> rows;
    std::map<int, ClassLaunch> cols;
    std::map<std::pair<int, int>, long long> widths;
    for (const HostSlot &h : b->host) {
        if (!h.used) continue;
        ClassLaunch &r = rows[std::make_pair(h.rows_key, h.prog)];
        r.smem = std::max(r.smem, h.rows_smem);
        r.items += h.rows_items;
        ClassLaunch &c = cols[h.cols_key];
        c.smem = std::max(c.smem, h.cols_smem);
        c.items += h.cols_items;
        for (int w : {1, 2, 4})
            if (h.pulse_items[w] > 0) widths[std::make_pair(h.kind, w)] += h.pulse_items[w];
    }
    BatchPlan p;
    for (const HostSlot &h : b->host) p.choppy = p.choppy || (h.used && h.choppy);
    p.rows.assign(rows.begin(), rows.end());
    p.cols.assign(cols.begin(), cols.end());
    p.widths.assign(widths.begin(), widths.end());
    return p;
}

extern "C" int ocs_batch_launches_per_step(const ocs_batch *b) {
    if (!b) return OCS_ERR_ARG;
    const BatchPlan p = batch_plan(b);
    return (int)(p.rows.size() + p.cols.size() + p.widths.size()) + 2 + (p.choppy ? 1 : 0);
}

extern "C" int ocs_batch_step(ocs_batch *b, int32_t pulses, void *stream) {
    if (!b || pulses < 0) return OCS_ERR_ARG;
    const BatchPlan p = batch_plan(b);
    BatchRef ref;
    ref.slots = b->d_slots;
    ref.nslots = 1;                           // slots past the last one in use hold nothing
    for (int i = 0; i < b->max_slots; ++i)
        if (b->host[i].used) ref.nslots = i + 1;
    cudaStream_t cs = (cudaStream_t)stream;
    for (int k = 0; k < pulses; ++k) {
        int st = OCS_OK;
        for (const auto &r : p.rows)
            if ((st = batch_launch_rows(ref, r.first.first, r.first.second, (int)r.second.items,
                                        (size_t)r.second.smem, cs)) != OCS_OK)
                return st;
        for (const auto &c : p.cols)
            if ((st = batch_launch_cols(ref, c.first, (int)c.second.items, (size_t)c.second.smem, cs)) != OCS_OK)
                return st;
        if (p.choppy && (st = batch_launch_choppy(ref, cs)) != OCS_OK) return st;
        if ((st = batch_launch_pulse_rows(ref, b->precision, cs)) != OCS_OK) return st;
        for (const auto &w : p.widths)
            if ((st = batch_launch_pulse(ref, b->precision, w.first.first, w.first.second, (int)w.second, cs)) !=
                OCS_OK)
                return st;
        batch_advance_kernel<<<1, 256, 0, cs>>>(ref);
        if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    }
    return OCS_OK;
}

extern "C" int ocs_batch_counters(const ocs_batch *b, int32_t *out, void *stream) {
    if (!b || !out) return OCS_ERR_ARG;
    std::vector<SlotState> h(b->max_slots);
    cudaStream_t cs = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(h.data(), b->d_slots, sizeof(SlotState) * b->max_slots,
                                    cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return OCS_ERR_CUDA;
    for (int s = 0; s < b->max_slots; ++s) out[s] = h[s].active ? h[s].counter : -1;
    return OCS_OK;
}

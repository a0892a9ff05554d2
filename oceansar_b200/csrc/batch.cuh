// Scene batch: many independent scenes advanced pulse by pulse by persistent kernels.
//
// Every scene of the batch occupies a slot.  Its static launch arguments (the SurfaceArgs
// and PulseArgs the single-scene entry points build) live in device memory, and so do its
// per-pulse tables (surface time, additive terms, azimuth position, Bragg refresh and
// scatterer offsets) and a pulse counter that the device advances at the end of every
// step.  One step = one pulse of every live scene: a persistent row-pass and column-pass
// kernel per transform length present, one row-table kernel, one fused pulse kernel per
// output-group width, and the counter advance.  Each persistent kernel enumerates its work
// items (row pairs, column tiles, facet tiles) over the slot table at run time, so the
// same sequence of launches -- and a CUDA graph recorded from it -- serves any set of
// scenes in the slots, and a step needs no host arguments.
#pragma once

#include "common.cuh"

namespace ocs {

constexpr int kMaxSlots = 256;

// Pulse-kernel classes of a slot: Kodis / Bragg scenes, and scenes with the Kirchhoff
// specular term (facet approach or stationary phase), which run their own instantiation.
constexpr int kSlotStd = 0;
constexpr int kSlotKa = 1;

// Flags of the per-pulse table.
constexpr int kFlagSurface = 1;     // synthesise the surface at this pulse
constexpr int kFlagRefresh = 2;     // refresh the Bragg RCS at this pulse

struct SlotState {
    int active;                     // 1 = in the batch
    int counter;                    // pulses done (advanced on the device)
    int az_steps;
    int nx, ny;
    int rows_key, cols_key;         // transform-length class of the row / column pass
    int npair;                      // packed transforms
    int nfields;
    int nout;                       // npol * nch
    int tile_rows;                  // rows per pulse-kernel tile
    int prog;                       // field program of the row pass
    int kind;                       // pulse-kernel class: kSlotStd or kSlotKa
    const float *t_tab;             // [az_steps] surface time (float32)
    const float *add_tab;           // [az_steps][nfields] additive field terms
    const float2 *swrot_tab;        // [az_steps] swell rotation exp(-i w_s t), or null
    const double *aznow_tab;        // [az_steps] platform azimuth position
    const int *flags_tab;           // [az_steps] kFlag*
    const int *tmod_tab;            // [az_steps][2] int(t prf) mod N_m, mod N_p
    const void *sargs;              // SurfaceArgs of the scene (device memory)
    const void *pargs;              // PulseArgs of the scene (device memory)
    const void *cargs;              // ChoppyArgs of a choppy scene (device memory), or null
};

struct BatchRef {
    SlotState *slots;
    int nslots;
};

// Work items of every slot for one kernel (count returns 0 for slots the kernel does not
// serve): writes the exclusive prefix over the slots into pref[0..nslots] and returns the
// total.  Warp 0 scans 32 slots per iteration with shuffles.  Every thread calls it.
template <class Count>
OCS_D int scan_slots(const BatchRef &b, int *pref, Count count) {
    if (threadIdx.x < 32) {
        int base = 0;
        for (int s0 = 0; s0 < b.nslots; s0 += 32) {
            const int s = s0 + (int)threadIdx.x;
            const int v = s < b.nslots ? count(b.slots[s]) : 0;
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += u;
            }
            if (s < b.nslots) pref[s] = base + incl - v;
            base += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (threadIdx.x == 0) pref[b.nslots] = base;
    }
    __syncthreads();
    return pref[b.nslots];
}

// Slot of item i: the last s with pref[s] <= i (binary search; uniform across the block).
OCS_D int find_slot(const int *pref, int nslots, int i) {
    int lo = 0, hi = nslots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// True when slot g takes part in the current step.
OCS_D bool slot_live(const SlotState &g) { return g.active && g.counter < g.az_steps; }

// ---- host-side pieces used by the batch engine (batch.cu) ----------------------------
size_t surface_args_bytes();
size_t pulse_args_bytes();
// Launch arguments of a scene as the single-scene entry points build them (time 0, the
// descriptor's pulse), written to out (surface_args_bytes() / pulse_args_bytes() bytes);
// prog receives the row pass's field program.
int surface_args_fill(const ocs_surface_desc *d, void *out, int *prog);
int pulse_args_fill(const ocs_pulse_desc *d, void *out);
// One launch over all slots of the batch: grid = the items of all slots in use of the
// class, one item per CTA (finished slots leave CTAs that return at once).
int batch_launch_rows(const BatchRef &b, int key, int prog, int grid, size_t smem, cudaStream_t st);
int batch_launch_cols(const BatchRef &b, int key, int grid, size_t smem, cudaStream_t st);
// Choppy surfaces: the slope / curvature step of every live choppy slot (after the column
// pass), its swell rotation taken from the slot's per-pulse table.
size_t choppy_args_bytes();
int choppy_args_fill(const ocs_choppy_desc *d, void *out);
int batch_launch_choppy(const BatchRef &b, cudaStream_t st);
int batch_launch_pulse_rows(const BatchRef &b, int precision, cudaStream_t st);
// Whether a scene's pulse descriptor takes the split-range mixed kernel (required of every
// Kodis / Bragg scene of a mixed-precision batch).
bool pulse_split_ok(const ocs_pulse_desc *d);
// Pulse-kernel class of a scene (kSlotStd / kSlotKa).
int pulse_kind(const ocs_pulse_desc *d);
int batch_launch_pulse(const BatchRef &b, int precision, int kind, int width, int grid, cudaStream_t st);
// Pulse-kernel items (groups of a width class x facet tiles) of one scene.
int batch_pulse_items(int nx, int ny, int tile_rows, int nout, int precision, int width);
// Row / column class key of a transform length (the length for compiled power-of-two
// lengths, 0 for the generic mixed-radix path); -1 if unsupported.
int surface_key(int n);
// Column tile width of a column class.
int surface_cols_tile(int key);
// Shared memory a row / column item of a class needs (bytes), -1 if it does not fit.
long long surface_rows_smem(int key, int nx);
long long surface_cols_smem(int key, int ny);

}  // namespace ocs

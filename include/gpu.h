// pcbroute search back end interface, as the router is compiled against it.
//
// This header declares the same types and functions as pcbroute's src/gpu.h:10-57 so that the router objects
// (router.cpp built with -DPCB_GPU) link against libpcbgpu unchanged. The member order and types of GpuQuery and
// GpuOut must stay exactly as they are: the router fills GpuQuery field by field (src/router.cpp:1527-1584) and
// reads GpuOut::best/rx0/ry0/rw/rh directly (src/router.cpp:1591-1600). Everything behind these declarations is
// the B200 implementation in pcbroute_b200/csrc (gpu_api.cpp over the pcbg_* C ABI of pcbg.h).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

// One search: the class's cost maps over the full grid (host arrays, layer by layer, [l][j * nx + i]), the search
// window inside it, the net's own copper overrides, the target bits, the optional learned prior and the starts.
// Replaces src/gpu.h:10-36 (same layout).
struct GpuQuery {
    int nx, ny, NL;                // full grid
    int wi0, wj0, ww, wh;          // search window (grid cells)
    uint16_t me;                   // the searching net as stored in the static grids (0 free, 0xFFFF blocked)
    float via_cost, step;          // via_cost < 0: vias not allowed; step: grid pitch (length unit of all costs)
    float dirf[8][8];              // per layer, cost factor of each of the 8 moves
    uint8_t lay[8];                // layers a track may use
    const float* cst[8];           // per layer cost map (>= 1e30: blocked; negative: someone's own copper)
    const uint16_t* st[8];         // per layer static owner grid
    const float* vcst;             // via-centre cost map
    const uint16_t* vst;           // via-centre static owner grid
    const uint64_t* tbit;          // target bits over window states (l * ww * wh + j * ww + i)
    std::vector<std::pair<uint32_t, float>> own_cf;   // window state -> resolved cost factor of the net's own cells
    std::vector<std::pair<uint32_t, float>> own_vcf;  // window cell -> resolved via factor of the net's own vias
    const uint8_t* prior = nullptr;                   // learned prior map (pnl x ph x pw bytes) or null
    int pi0 = 0, pj0 = 0, pw = 0, ph = 0, pnl = 0;
    const int* pcol = nullptr;                        // full-grid column -> prior pixel column
    const int* prow = nullptr;                        // full-grid row -> prior pixel row
    int play[8];                                      // router layer -> prior layer (-1: none)
    float mlf[256];                                   // cost factor per prior value
    uint8_t mthr = 0;                                 // corridor threshold
    bool corridor = false;
    std::vector<std::pair<uint32_t, float>> starts;   // window state, initial cost
};

// The solved part of the window: a rectangle of it with the cost of every state (1e30 where it is not reached
// at or below the cheapest target), and the cheapest target. Replaces src/gpu.h:39-50 (same layout).
struct GpuOut {
    int rx0 = 0, ry0 = 0, rw = 0, rh = 0, NL = 0, ww = 0, wh = 0;
    int64_t best = -1;                   // cheapest target as a window state, -1 if none can be reached
    float* d = nullptr;                  // pinned host buffer, [l][j][i] over the rectangle
    size_t cap = 0;
    GpuOut() = default;
    GpuOut(const GpuOut&) = delete;
    GpuOut& operator=(const GpuOut&) = delete;
    ~GpuOut();
    void reserve(size_t n);
    float operator()(int64_t q) const;   // cost of a window state
};

// src/gpu.h:52 -- true when a usable B200 is present.
bool gpu_available();
// src/gpu.h:53-54 -- how many solves may be in flight at once, and the most states one solve may take.
void gpu_configure(int slots, size_t max_states);
// src/gpu.h:55-57 -- solve one search. Returns the relaxation rounds it took (>= 1), -1 on failure (the router then
// carries on with its CPU search), -3 if every slot is busy and wait is false.
int gpu_solve(const GpuQuery& q, GpuOut& out, bool wait = true);

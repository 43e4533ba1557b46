// Host-side plan structures and kernel launch tables.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "rk_params.h"

namespace rk {

enum PassKind { PK_LINE = 0, PK_PLANE = 1 };
enum BufId { BUF_IN = -1, BUF_OUT = -2 };

using LineLaunch = cudaError_t (*)(const PassParams&, int64_t nblocks, cudaStream_t);
using PlaneLaunch = cudaError_t (*)(const PassParams&, int64_t nplanes, cudaStream_t);

struct LineInfo {
    LineLaunch fn;
    int nt;        // threads per CTA
    int nl;        // lines per CTA
    size_t smem;   // dynamic shared memory bytes
};

struct TmaInfo {
    LineLaunch fn;
    int (*per_sm)();   // resident CTAs per SM
    int nt;
    int nl;
    size_t smem;
};
// persistent TMA-fed plain line pass of length L and mode
bool tma_info(int dbl, int L, int mode, TmaInfo* out);
bool encode_lane_map(void* base, int dbl, int64_t I, int64_t L, int64_t O, int64_t sj, int64_t so, int nl, int rows,
                     TensorMapBytes* out);

struct PlaneTmaInfo {
    LineLaunch fn;        // nblocks = CTAs of the persistent grid
    int (*clusters)();    // clusters resident at once
    int q;
    int nt;
    size_t smem;
};
bool plane_tma_info(int dbl, int L1, int L2, PlaneTmaInfo* out);

struct PlaneInfo {
    PlaneLaunch fn;
    int q;         // cluster size
    int nt;
    size_t smem;
};

// lookup; returns false if the combination is not compiled
bool line_info(int dbl, int L, int mode, int var, LineInfo* out);
// fused Bluestein pass on a two-CTA cluster a line (variant 7, rk_blue2.cu); L = M/2
bool blue2_info(int dbl, int L, LineInfo* out);
bool plane_info(int dbl, int L1, int L2, int wide, PlaneInfo* out);

// row + column passes of a plane in one persistent launch (rk_pair.cu)
struct PairInfo {
    cudaError_t (*launch)(const void* args, cudaStream_t st);
    int (*resident)();   // CTAs resident at once on the device
    int nl_rows, nl_cols;
};

struct PassRec {
    int kind = PK_LINE;
    int dbl = 0;
    int L = 0, mode = 0;
    int var = 0;                   // 0 plain, 1 fused Bluestein, 2 transposed store
    bool blue = false;
    int L1 = 0, L2 = 0;            // plane
    int axis = -1, axis2 = -1;
    int ld_buf = BUF_IN, st_buf = BUF_OUT;
    bool ld_edge = false, st_edge = false;
    bool inplace_safe = true;      // each CTA rewrites only what it read
    PassParams prm{};
    PlaneParams pprm{};
    int64_t nblocks = 0;
    LineInfo li{};
    PlaneInfo pi{};
    TmaInfo ti{};
    PlaneTmaInfo pti{};
    bool use_plane_tma = false;
    int64_t plane_tma_blocks = 0;
    bool use_tma = false;
    bool use_tc = false;           // tensor-core split-precision kernel (RK_FLAG_SPLIT_TC)
    bool pair_first = false;       // this pass and the next run as one pair launch
    PairInfo pair{};
    void* pair_tasks = nullptr;    // int32 task table
    void* pair_counters = nullptr; // task counter + per-plane row-tile counters
    int64_t pair_ntasks = 0, pair_planes = 0;
    int32_t pair_a = 0, pair_b = 0;
    int user_bits = 0;             // 1: loads an RK_FMT_USER input edge, 2: stores one
    void* user_lib = nullptr;      // cudaLibrary_t of the installed run-time compiled kernel
    const void* user_kern = nullptr;  // its cudaKernel_t
    bool tma_reencode = false;     // tensor map over the user's input: re-encode per call
    const void* tma_ptr = nullptr; // pointer the current map was encoded for
    int tma_rows = 0;
    std::string note;
};

bool pair_info(int dbl, int LR, int LC, PairInfo* out);
int pair_setup(PassRec& ra, PassRec& rb, const PairInfo& pi);
cudaError_t pair_launch(const PassRec& ra, const PassParams& pa, const PassParams& pb, int32_t* status,
                        cudaStream_t st);

// tensor-core split-precision pass (rk_tc.cu): 256- and 1024-point complex64
// contiguous lines; tc_prepare generates its tables on the current device (once)
bool tc_eligible(const PassRec& r);
cudaError_t tc_prepare();
cudaError_t tc_launch(const PassParams& p, int L, cudaStream_t st);

struct DeviceTables {
    void* stw_f = nullptr;     // float2 stage twiddle tables, all L (TwLayout)
    void* stw_d = nullptr;     // double2 stage twiddle tables
    int64_t off_f[16] = {0};   // element offset of the table of L = 2^i
    int64_t off_f_r16 = 0;     // the 16-element plan of L = 8192 (RadixP<float, 8192, 1>)
    int64_t off_d[16] = {0};
    int64_t bytes = 0;
    void* tw4hi_f = nullptr;   // float2[4096]
    void* tw4lo_f = nullptr;
    void* tw4hi_d = nullptr;   // double2[4096]
    void* tw4lo_d = nullptr;
    int32_t* status = nullptr; // device status word
};

// per-device twiddle tables, generated once on the device in FP64
int device_tables(int device, DeviceTables** out);

void set_error(const std::string& msg);

}  // namespace rk

struct rk_fft_plan {
    int device = 0;
    rk_fft_desc desc{};
    std::vector<rk::PassRec> passes;
    std::vector<void*> temps;
    std::vector<int64_t> temp_bytes;
    std::vector<void*> tables;
    int64_t device_bytes = 0;
    double n_total = 1.0;          // inverse normalisation
    bool alias_hazard = false;     // single remapping pass: in == out needs a copy
    void* alias_tmp = nullptr;
    int64_t in_extent_bytes = 0;   // bytes spanned by the input array (alias copy)
    int64_t in2_extent_bytes = 0;
    // per-pass event profiling (rk_fft_profile)
    std::vector<cudaEvent_t> prof_ev;   // 2 * passes * max_calls
    int32_t prof_max = 0, prof_used = 0;
};

// Host-side launch interface of the wavefront kernels (wr_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "wr_device.cuh"
#include "wr_guide.h"

namespace wrk {

using namespace wrd;

struct WaveBuffers {
    float4 *o[2], *d[2], *thr[2];
    uint32_t *meta[2];
    uint32_t *rec[2];                  // per-slot training record (guided renders that collect records)
    float4 *hit;
    float4 *sh_o, *sh_d, *sh_c;
    double *film;                      // base (npix*3) then splat (npix*3)
    uint32_t *ctr;                     // CTR_COUNT counters
    unsigned long long *sample_next;
    uint32_t capacity, shadow_capacity;
    uint4 *lobes;                      // packed lobes, wrg::kPackedChunks x capacity (guided renders)
    float4 *records;                   // training records
    uint32_t *rec_count;
    uint32_t rec_capacity;
};

struct RenderLaunch {
    const wrd::DevJob *jobs;    // device job table (nullptr: the single job `job0`)
    wrd::DevJob job0;
    int num_jobs;
    uint32_t total_pix;         // film pixels over all jobs
    unsigned long long total_samples;
    uint32_t iter_limit;        // the loop stops (and reports CTR_TIMEOUT) after this many iterations
    int grid_trace, grid_shade;
    int trace_block;            // threads per block of extend / shadow: 64, 128 or 256
    cudaGraphConditionalHandle cond;   // while-loop condition when the loop body is captured in a graph
    int has_cond;
    unsigned long long *prof;   // device profiling totals or nullptr
    const wrg::GuideNet *guide; // learned proposal used by shade (nullptr: plain NEE+MIS)
    int record;                 // 1: collect training records
    int guide_sms;              // SM count (grid of the inference kernel)
    int fetch_min;              // dynamic ray fetching threshold (lanes still traversing)
    int nee_only;               // 1: every job is nextevent_path_tracer (shade without the other
                                // integrators' branches); 0: any mix of integrators
};

enum KernelId { KERNEL_EXTEND = 0, KERNEL_SHADE = 1, KERNEL_RAYGEN = 2, KERNEL_SHADOW = 3, KERNEL_ADVANCE = 4,
                KERNEL_RESOLVE = 5, KERNEL_GUIDE = 6,
                // fused schedule: extend + the previous iteration's shadow rays; the last shadow rays
                KERNEL_TRACE_PAIR = 8, KERNEL_SHADOW_FLUSH = 9 };

void launch_kernel(int which, const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity,
                   cudaStream_t st);
void launch_prime(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st);
void launch_iteration(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity, cudaStream_t st);
// fused schedule: extend + the previous iteration's shadow rays in one launch, then a flush of
// the last iteration's shadow rays after the loop
void launch_prime_fused(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st);
void launch_iteration_fused(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity,
                            cudaStream_t st);
void launch_shadow_flush(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st);
void launch_resolve(const double *film, double *out, const RenderLaunch &r, cudaStream_t st);
void launch_trace_batch(const DevScene &s, const float4 *rays, uint32_t n, int any_hit, float4 *out, uint32_t *visits,
                        int grid, cudaStream_t st);
void launch_cdf_build(const double *weights, const uint32_t *offsets, uint32_t ntables, float *cdf, float *pdf,
                      double *sums, cudaStream_t st);
void launch_env_weights(const float4 *texels, int w, int h, double *out, cudaStream_t st);
void launch_scale_pdf(const double *weights, double total, float *pdf, size_t n, cudaStream_t st);
// resident blocks per SM of the extend (which 0; the variant for Phong patches and / or the
// compressed 8-wide BVH) or shade (which 1) kernel
int occupancy_blocks(int which, int trace_block = 128, bool phong = false, bool wide = false);

}  // namespace wrk

// ref_shims.cu -- extern "C" launchers around the reference's own CUDA kernels, for the benchmark's
// comparator sections only (never linked into the product library).
//
// oracle/build_ref.py compiles this file once per kernel family, passing the path of the reference source
// file in REF_SOURCE; the reference source is included unmodified, and its program's main() is renamed by
// the command line (-Dmain=...) so that the translation unit links as a shared library.  Each launcher uses
// the launch shape of the reference's own host code:
//   REF_AWR        mat_vec_ans_warp_per_row   buffered/ans-warp-rows-kernel.cu:7-221,
//                  launched as in buffered/ans-warp-rows.cu:50-57 (one 32-thread block per row)
//   REF_DENSE      vecMat_int8_warpRows       baselines/baseline_int8/baseline_matVec_custom.cu:99-155,
//                  launched as in baseline_matVec_custom.cu:407-412 (4 warps per block)
//   REF_WPR        decmpressAndMultiply       matvansWarpPerRow/matvansWarpPerRow-kernel.cu:46-175,
//                  launched as in matvansWarpPerRow/matvansWarpPerRow.cu:150-164
//   REF_WPR_LOCAL  decmpressAndMultiply       matvansWarpPerRow/matvansWarpPerRow_local_cdf.cu:196-334
//                  (cdf in constant memory, uploaded as in :478), launched as in :336-351
// Every launcher returns the cudaError_t of its launch.  Known over-reads of these kernels (the refill of
// the last row's stream reads past it) must land inside the caller's allocations: the benchmark pads every
// stream buffer.
#include <cstdint>
#include <cuda_runtime.h>

#include REF_SOURCE

#if defined(REF_AWR)
extern "C" int ref_awr_launch(void *out8, const void *compressed, const uint32_t *warp_offsets, const uint32_t *ppf,
                              const uint32_t *ppf_cum, const uint32_t *ppf_prob, const void *x, int in_dim,
                              int out_dim, float scale, void *stream) {
    mat_vec_ans_warp_per_row<<<out_dim, 32, in_dim, (cudaStream_t)stream>>>(
        reinterpret_cast<uint4 *>(out8), reinterpret_cast<const uint4 *>(compressed), warp_offsets, ppf, ppf_cum,
        ppf_prob, reinterpret_cast<const uint4 *>(x), in_dim, out_dim, scale);
    return (int)cudaGetLastError();
}
#elif defined(REF_DENSE)
extern "C" int ref_dense_launch(int32_t *y, const int8_t *W, const int8_t *x, int cols, int rows, void *stream) {
    const int warps_per_block = 4;
    vecMat_int8_warpRows<<<(rows + warps_per_block - 1) / warps_per_block, warps_per_block * 32, cols,
                           (cudaStream_t)stream>>>(y, W, x, cols, rows);
    return (int)cudaGetLastError();
}
#elif defined(REF_WPR) || defined(REF_WPR_LOCAL)
extern "C" int ref_wpr_launch(int32_t *y, int8_t *x, uint32_t rows, uint32_t cols, const uint32_t *cursors,
                              int8_t min_value, uint8_t G, const uint8_t *cdf, const uint8_t *ppf,
                              uint16_t *payload, uint32_t payload_size, void *stream) {
    const int warps_per_block = 4;
    const dim3 grid((rows + warps_per_block - 1) / warps_per_block), block(warps_per_block * 32);
#if defined(REF_WPR_LOCAL)
    // the variant reads its cdf from constant memory (matvansWarpPerRow_local_cdf.cu:18, :478)
    cudaError_t e = cudaMemcpyToSymbolAsync(d_cdf_data, cdf, (size_t)G + 1, 0, cudaMemcpyDeviceToDevice,
                                            (cudaStream_t)stream);
    if (e != cudaSuccess) return (int)e;
    decmpressAndMultiply<<<grid, block, ((size_t)G + 1) * sizeof(int32_t), (cudaStream_t)stream>>>(
        y, x, rows, cols, 1.0f, cursors, min_value, G, cdf, ppf, payload, payload_size);
#else
    decmpressAndMultiply<<<grid, block, cols, (cudaStream_t)stream>>>(y, x, rows, cols, 1.0f, cursors, min_value, G,
                                                                      cdf, ppf, payload, payload_size);
#endif
    return (int)cudaGetLastError();
}
#endif

// Registry of the compiled kernel variants (precision x threads-per-lane x largest column tier).
// Every variant object file registers its two kernels at load time; the C ABI looks them up.
#pragma once

namespace pe {

void register_variant(int mixed, int tpl, int kpm, void* chain_kernel, void* cofactor_kernel, void* split_partial,
                      void* split_draw, void* warp_kernel, size_t warp_slice_bytes);
void* find_chain_kernel(int mixed, int tpl, int kpm);
void* find_cofactor_kernel(int mixed, int tpl, int kpm);
void* find_split_partial_kernel(int mixed, int tpl, int kpm);
void* find_split_draw_kernel(int mixed, int tpl, int kpm);
void* find_warp_kernel(int mixed, int tpl, int kpm);
size_t warp_smem_bytes(int mixed, int tpl, int kpm, int warps);   // the variant's slice per stream x warps

}  // namespace pe

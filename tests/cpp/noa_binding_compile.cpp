// Compile check (not linked): the reference-side binding instantiates against noa's own types for
// every function, with Views, constant values, Empty weights, Mat22/Mat33/Quaternion values and arrays.
#include "noa_b200/noa_binding.hpp"

using namespace ::noa::types;
namespace nx = ::noa::xform;
namespace bind = ::noa_b200::binding;

void instantiate(View<const c32> vol, View<const f32> volw, View<c32> slices, View<f32> slices_w,
                 View<f32> slices_real, View<const Mat33<f32>> rot, View<const nx::Quaternion<f32>> quat,
                 View<const Mat22<f32>> scale, View<const c32> in_slices, View<c32> grid, View<f32> grid_w,
                 void* stream) {
    const Shape4 vshape{1, 8, 8, 8}, sshape{2, 1, 8, 8};
    bind::extract<"hc2h">(vol, Empty{}, vshape, slices, Empty{}, sshape, Empty{}, rot,
                          nx::ExtractCentralSlicesOptions{}, stream);
    bind::extract<"h2hc">(vol, volw, vshape, slices_real, slices_w, sshape, scale, quat,
                          nx::ExtractCentralSlicesOptions{.interp = nx::Interp::LANCZOS8}, stream);
    bind::extract<"hc2hc">(vol, Empty{}, vshape, slices, Empty{}, sshape, Mat22<f32>::eye(1), Mat33<f32>::eye(1),
                           nx::ExtractCentralSlicesOptions{}, stream);
    bind::rasterize<"h2hc">(in_slices, Empty{}, sshape, grid, grid_w, vshape, Empty{}, rot,
                            nx::RasterizeCentralSlicesOptions{}, stream);
    bind::rasterize<"hc2h">(c32{1, 2}, f32{1}, sshape, grid, grid_w, vshape, Empty{}, nx::Quaternion<f32>{0, 0, 0, 1},
                            nx::RasterizeCentralSlicesOptions{.fftfreq_cutoff = 0.45}, stream);
    bind::insert<"hc2hc">(in_slices, Empty{}, sshape, grid, grid_w, vshape, Empty{}, rot,
                          nx::InsertCentralSlicesOptions{.windowed_sinc = {-1, 0.05}}, stream);
    bind::insert_and_extract<"hc2h">(in_slices, Empty{}, sshape, slices, slices_w, sshape, Empty{}, rot, scale, quat,
                                     nx::InsertAndExtractCentralSlicesOptions{.correct_weights = true}, stream);
}

// Texture inputs (staged into linear memory by the binding; with NOA_ENABLE_CUDA through the CUDA array).
void instantiate_textures(const nx::Texture<c32>& tvol, const nx::Texture<f32>& tvolw, const nx::Texture<c32>& tslices,
                          View<c32> slices, View<f32> slices_w, View<const Mat33<f32>> rot, View<c32> grid,
                          View<f32> grid_w, void* stream) {
    const Shape4 vshape{1, 8, 8, 8}, sshape{2, 1, 8, 8};
    bind::extract<"hc2h">(tvol, tvolw, vshape, slices, slices_w, sshape, Empty{}, rot,
                          nx::ExtractCentralSlicesOptions{}, stream);
    bind::insert<"hc2hc">(tslices, Empty{}, sshape, grid, grid_w, vshape, Empty{}, rot,
                          nx::InsertCentralSlicesOptions{}, stream);
    bind::insert_and_extract<"hc2h">(tslices, Empty{}, sshape, slices, slices_w, sshape, Empty{}, rot, Empty{}, rot,
                                     nx::InsertAndExtractCentralSlicesOptions{}, stream);
}

// Placeholder launchers for the stages not yet on the device.
#include "../../include/pxl.h"
#include "pxl_internal.cuh"
namespace pxl {
void launch_fit(const Dev&, const Launch&) {}
void launch_classify(const Dev&, const Launch&) {}
void launch_vertices(const Dev&, const Launch&) {}
}  // namespace pxl
extern "C" int32_t pxl_bl_fit(const double*, const float*, const int32_t*, int32_t, double, int32_t, float*, float*,
                              float*, float*, float*, int32_t*, void*) { return PXL_ERR_STATE; }

// Generated by cardioid_b200/data/make_fit_shapes.py from the shipped
// dt = 0.02 BetterTT06 fit files; do not edit.
#pragma once
namespace cdb {
constexpr int kSpecNumer[30] = {3, 10, 6, 11, 4, 9, 6, 7, 6, 11, 5, 9, 6, 19, 8, 19, 8, 12, 5, 7, 7, 12, 7, 6, 3, 7, 4, 5, 7, 9};
constexpr int kSpecDenom[30] = {3, 7, 5, 1, 3, 9, 3, 11, 5, 13, 6, 16, 5, 14, 5, 13, 5, 14, 5, 7, 5, 12, 5, 1, 5, 3, 7, 3, 12, 14};
constexpr int kSpecOffset[30] = {0, 5, 21, 31, 42, 48, 65, 73, 90, 100, 123, 133, 157, 167, 199, 211, 242, 254, 279, 288, 301, 312, 335, 346, 352, 359, 368, 378, 385, 403};
constexpr int kSpecPool = 425;
// FP32 form of the mixed kernels: fits in kSpecShiftMask take t = (x - kSpecShift) / kSpecShiftScale
constexpr float kSpecShift[30] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, -40.0f, -90.0f, 0.0f, -90.0f, -70.0f, 0.0f, 0.0f, 0.0f, -15.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 40.0f, -20.0f};
constexpr float kSpecShiftScale = 128.0f;
constexpr unsigned kSpecShiftMask = 0x30236000u;
}  // namespace cdb

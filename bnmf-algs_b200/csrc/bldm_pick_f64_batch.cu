// Instantiations of the multi-instance F64 sweep kernels by lane shape.
#include "bldm_sweep_kernels.cuh"

namespace bldm {

#define BLDM_SHAPE_CASES(T, VEC, UPD, APPR, MR, CP)                                        \
    case 1 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 1, 1, UPD, APPR, MR, CP>); \
    case 2 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 2, 1, UPD, APPR, MR, CP>); \
    case 4 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 4, 1, UPD, APPR, MR, CP>); \
    case 8 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 8, 1, UPD, APPR, MR, CP>); \
    case 16 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 16, 1, UPD, APPR, MR, CP>); \
    case 32 * 16 + 1: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 32, 1, UPD, APPR, MR, CP>); \
    case 32 * 16 + 2: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 32, 2, UPD, APPR, MR, CP>); \
    case 32 * 16 + 4: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 32, 4, UPD, APPR, MR, CP>); \
    case 32 * 16 + 8: return reinterpret_cast<void*>(&sweep_batch_kernel<T, VEC, 32, 8, UPD, APPR, MR, CP>);

template <typename T, int VEC, bool UPD, bool APPR, bool MR, bool CP>
static void* shape_case(int lpf, int mch) {
    switch (lpf * 16 + mch) { BLDM_SHAPE_CASES(T, VEC, UPD, APPR, MR, CP) default: return nullptr; }
}

// mode: 0 axis sums, 1 update, 2 compact update (listed rows only).
template <typename T, int VEC, bool APPR>
static void* shape(int lpf, int mch, bool mr, int mode) {
    if (mode == 0)
        return mr ? shape_case<T, VEC, false, true, true, false>(lpf, mch)
                  : shape_case<T, VEC, false, true, false, false>(lpf, mch);
    if (mode == 1)
        return mr ? shape_case<T, VEC, true, APPR, true, false>(lpf, mch)
                  : shape_case<T, VEC, true, APPR, false, false>(lpf, mch);
    return mr ? shape_case<T, VEC, true, APPR, true, true>(lpf, mch)
              : shape_case<T, VEC, true, APPR, false, true>(lpf, mch);
}

void* pick_sweep_f64_batch(int vec, int lpf, int mch, int mode, bool appr, bool mr) {
    if (vec == 2)
        return appr ? shape<double, 2, true>(lpf, mch, mr, mode)
                    : shape<double, 2, false>(lpf, mch, mr, mode);
    return appr ? shape<double, 1, true>(lpf, mch, mr, mode)
                : shape<double, 1, false>(lpf, mch, mr, mode);
}

}  // namespace bldm

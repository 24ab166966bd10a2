// Instantiations of the single-instance F64 sweep kernels by lane shape.
#include "bldm_sweep_kernels.cuh"

namespace bldm {

#define BLDM_SHAPE_CASES(T, VEC, UPD, APPR, MR)                                                \
    case 1 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 1, 1, UPD, APPR, MR>);       \
    case 2 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 2, 1, UPD, APPR, MR>);       \
    case 4 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 4, 1, UPD, APPR, MR>);       \
    case 8 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 8, 1, UPD, APPR, MR>);       \
    case 16 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 16, 1, UPD, APPR, MR>);     \
    case 32 * 16 + 1: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 32, 1, UPD, APPR, MR>);     \
    case 32 * 16 + 2: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 32, 2, UPD, APPR, MR>);     \
    case 32 * 16 + 4: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 32, 4, UPD, APPR, MR>);     \
    case 32 * 16 + 8: return reinterpret_cast<void*>(&sweep_kernel<T, VEC, 32, 8, UPD, APPR, MR>);

template <typename T, int VEC, bool UPD, bool APPR, bool MR>
static void* shape_case(int lpf, int mch) {
    switch (lpf * 16 + mch) { BLDM_SHAPE_CASES(T, VEC, UPD, APPR, MR) default: return nullptr; }
}

template <typename T, int VEC, bool UPD, bool APPR>
static void* shape(int lpf, int mch, bool mr) {
    return mr ? shape_case<T, VEC, UPD, APPR, true>(lpf, mch)
              : shape_case<T, VEC, UPD, APPR, false>(lpf, mch);
}

void* pick_sweep_f64_plain(int vec, int lpf, int mch, bool update, bool appr, bool mr) {
    if (vec == 2) {
        if (!update) return shape<double, 2, false, true>(lpf, mch, mr);
        return appr ? shape<double, 2, true, true>(lpf, mch, mr)
                    : shape<double, 2, true, false>(lpf, mch, mr);
    }
    if (!update) return shape<double, 1, false, true>(lpf, mch, mr);
    return appr ? shape<double, 1, true, true>(lpf, mch, mr)
                : shape<double, 1, true, false>(lpf, mch, mr);
}

}  // namespace bldm

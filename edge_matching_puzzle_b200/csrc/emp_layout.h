// Constants shared by the host table builder (emp_model.cpp) and the kernels.
#pragma once

#include <cstdint>

namespace emp {

// 32-bit words per level descriptor in a puzzle's table blob (see emp_model.h)
constexpr uint32_t kDescWords = 16;

// Where the exhaustive DFS keeps its stack, and who walks it (emp_bt.cu)
enum StackMode : int {
    kStackShared32 = 1,  // shared memory, 32-bit entries holding the placed piece's colours
    kStackShared16 = 2,  // shared memory, 16-bit entries (colours read from the transition table)
    kStackGlobal32 = 3,  // global memory (L1-cached), 32-bit entries
    kStackWarp = 4,      // one DFS per warp: the warp's stack in shared memory, a candidate word per lane
};

}  // namespace emp

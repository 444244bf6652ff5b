// Project-written stand-in for FSM_base::FSM_context<TRANSITION> (external FSM
// framework of the reference).  emp_FSM_context only derives from it.
#pragma once

#include <string>

namespace FSM_base {
template <typename TRANSITION>
class FSM_context {
  public:
    FSM_context() = default;
    virtual ~FSM_context() = default;
};
}  // namespace FSM_base

// Project-written stand-in for FSM_interfaces::FSM_transition_if (external
// FSM framework of the reference).  Test infrastructure for oracle/_ref.
#pragma once

#include <string>

namespace FSM_interfaces {
class FSM_transition_if {
  public:
    virtual const std::string to_string() const = 0;
    virtual void to_string(std::string&) const = 0;
    virtual ~FSM_transition_if() = default;
};
}  // namespace FSM_interfaces

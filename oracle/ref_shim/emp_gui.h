// Project-written stand-in that shadows the reference's include/emp_gui.h (an SDL
// window, off the search path).  emp_strategy calls display() and refresh() on
// "New max"; here they do nothing.  Test infrastructure for oracle/_ref.
#ifndef EMP_GUI_H
#define EMP_GUI_H

#include "emp_FSM_situation.h"

namespace edge_matching_puzzle {
class emp_gui {
  public:
    emp_gui() = default;
    void display(const emp_FSM_situation&) {}
    void refresh() {}
};
}  // namespace edge_matching_puzzle

#endif

// Project-written stand-in for FSM_base::FSM_situation<CONTEXT> and
// FSM_interfaces::FSM_situation_if (external FSM framework of the reference).
// emp_FSM_situation uses get_context() / set_context(); the situation owns the
// context it is given (include/emp_strategy.h creates it with new).
#pragma once

#include <string>

namespace FSM_interfaces {
class FSM_situation_if {
  public:
    virtual const std::string to_string() const = 0;
    virtual const std::string get_string_id() const = 0;
    virtual void to_string(std::string&) const = 0;
    virtual void get_string_id(std::string&) const = 0;
    virtual bool is_final() const = 0;
    virtual bool less(const FSM_situation_if*) const = 0;
    virtual ~FSM_situation_if() = default;
};
}  // namespace FSM_interfaces

namespace FSM_base {
template <typename CONTEXT>
class FSM_situation : public FSM_interfaces::FSM_situation_if {
  public:
    FSM_situation() : m_context(nullptr) {}
    FSM_situation(const FSM_situation& o) : m_context(o.m_context ? new CONTEXT(*o.m_context) : nullptr) {}
    ~FSM_situation() override { delete m_context; }
    CONTEXT* get_context() const { return m_context; }
    void set_context(CONTEXT& c)
    {
        if (m_context != &c) delete m_context;
        m_context = &c;
    }

  private:
    CONTEXT* m_context;
};
}  // namespace FSM_base

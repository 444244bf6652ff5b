// Project-written stand-in for the reference's external quicky_exception
// library: exceptions carrying a message, a line and a file
// (use: src/main.cpp:137-146).  Test infrastructure for oracle/_ref.
#pragma once

#include <stdexcept>
#include <string>

namespace quicky_exception {

class quicky_base_exception {
  public:
    quicky_base_exception(const std::string& m, unsigned int line, const std::string& file)
        : m_msg(m), m_line(line), m_file(file) {}
    virtual ~quicky_base_exception() = default;
    const char* what() const noexcept { return m_msg.c_str(); }
    unsigned int get_line() const { return m_line; }
    const std::string& get_file() const { return m_file; }

  private:
    std::string m_msg;
    unsigned int m_line;
    std::string m_file;
};

class quicky_logic_exception : public quicky_base_exception, public std::logic_error {
  public:
    quicky_logic_exception(const std::string& m, unsigned int line, const std::string& file)
        : quicky_base_exception(m, line, file), std::logic_error(m) {}
    const char* what() const noexcept override { return quicky_base_exception::what(); }
};

class quicky_runtime_exception : public quicky_base_exception, public std::runtime_error {
  public:
    quicky_runtime_exception(const std::string& m, unsigned int line, const std::string& file)
        : quicky_base_exception(m, line, file), std::runtime_error(m) {}
    const char* what() const noexcept override { return quicky_base_exception::what(); }
};

}  // namespace quicky_exception

// C++ host layer over the C ABI of include/emp_b200.h.
//
// It mirrors the reference's plugin interface for its two GPU searches, with the
// same class names, constructor arguments and error behaviour, so that a program
// written against the reference's features reads the same here:
//
//   feature_if                  include/feature_if.h:27-33
//   feature_CUDA_backtracker    include/feature_CUDA_backtracker.h:33-72,
//                               src/feature_CUDA_backtracker.cpp:31-38
//   feature_CUDA_glutton_max    include/feature_CUDA_glutton_max.h:31-75
//   factory_feature             include/factory_feature.h:142-164
//   emp_pieces_parser::parse    include/emp_pieces_parser.h:53-101
//   strategy generators         include/emp_basic_strategy_generator.h:44-53 (basic),
//                               include/emp_spiral_strategy_generator.h:52-100 (spiral)
//   board strings               include/situation_string_formatter.h:51-70
//
// Where the reference throws quicky_exception::quicky_logic_exception, this layer
// throws emp_logic_error with the same what()/file/line triple; the CLI (main.cpp)
// catches it and exits with -1 as src/main.cpp:137-146 does.
#pragma once

#include "emp_b200.h"

#include <cstdint>
#include <iostream>
#include <istream>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace edge_matching_puzzle {

class emp_logic_error : public std::logic_error {
  public:
    emp_logic_error(const std::string& what, unsigned line, const char* file)
        : std::logic_error(what), m_line(line), m_file(file)
    {
        const size_t slash = m_file.find_last_of('/');  // keep the file name only
        if (slash != std::string::npos) m_file.erase(0, slash + 1);
    }
    unsigned get_line() const { return m_line; }
    const std::string& get_file() const { return m_file; }

  private:
    unsigned m_line;
    std::string m_file;
};

// Pieces of a puzzle definition file: colours[4*(id-1)+side], sides N,E,S,W, 0 = frame.
struct emp_piece_set {
    uint32_t width = 0;
    uint32_t height = 0;
    std::vector<uint8_t> colours;
    uint32_t size() const { return static_cast<uint32_t>(colours.size() / 4); }
};

// Reads the reference's CSV puzzle format ("Width,Height" / "w,h" / "I,N,E,S,O" / one
// line per piece).  Throws emp_logic_error on an unreadable or malformed file.
emp_piece_set parse_pieces(const std::string& path);

// Visiting order of the positions (the reference's emp_strategy_generator).
class emp_strategy_generator {
  public:
    emp_strategy_generator(std::string name, uint32_t width, uint32_t height, std::vector<uint16_t> order)
        : m_name(std::move(name)), m_width(width), m_height(height), m_order(std::move(order)) {}
    const std::string& get_name() const { return m_name; }
    // (x, y) of the index-th visited position
    std::pair<unsigned, unsigned> get_position(unsigned index) const
    {
        return {m_order.at(index) % m_width, m_order.at(index) / m_width};
    }
    const std::vector<uint16_t>& order() const { return m_order; }
    uint32_t get_width() const { return m_width; }
    uint32_t get_height() const { return m_height; }

  private:
    std::string m_name;
    uint32_t m_width, m_height;
    std::vector<uint16_t> m_order;
};

// "basic" (row major), "spiral", or else the name of a text strategy file, as
// emp_strategy_generator_factory::create does (src/emp_strategy_generator_factory.cpp:
// 24-39).  A text strategy (include/emp_text_strategy_generator.h:66-107) lists one
// "x,y" position per line in visiting order; empty lines and lines starting with '#'
// are skipped.  Throws emp_logic_error on a malformed or incomplete file, and when the
// order does not list every position once.
std::unique_ptr<emp_strategy_generator> create_strategy_generator(const std::string& name, uint32_t width,
                                                                  uint32_t height);

// The stream strategy (include/emp_stream_strategy_generator.h): width*height (x, y)
// pairs of 32-bit little-endian words read from a binary stream, the form in which a
// results.bin file stores the order it was written with.
std::unique_ptr<emp_strategy_generator> read_stream_strategy(std::istream& in, uint32_t width, uint32_t height);

// Transitions (kind_index << 2 | orientation) of a situation string's pieces along
// the strategy's order, up to its first empty position (include/emp_strategy.h:
// 431-441 with include/situation_string_formatter.h:80-121).  Throws emp_logic_error
// on a malformed string.
std::vector<uint16_t> situation_transitions(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                                            const std::string& situation);

// The reference's board string: per position y*w+x the piece id right-aligned on
// digits(w*h) characters plus N/E/S/W, or dashes when empty.  cells[pos] holds
// (id-1)<<2 | orientation, or 0xFFFFFFFF when empty.
std::string situation_string(uint32_t width, uint32_t height, const uint32_t* cells);

class feature_if {
  public:
    virtual void run() = 0;
    virtual ~feature_if() = default;
};

// Settings the reference hard-codes; the defaults reproduce its behaviour.
struct feature_options {
    std::string initial_situation;  // new_strategy, CUDA_backtracker: resume from this situation string
    bool trace = false;             // CUDA_backtracker: the reference's variable-space search and its trace
    bool stop_at_first = false;     // backtracker: stop at the first solution found
    uint32_t split_depth = 0;       // backtracker: 0 = library default
    uint64_t push_budget = 0;       // glutton: stop after this many placements (0 = none)
    uint32_t timeout_ms = 0;        // 0 = library default
    int device = -1;                // CUDA device, -1 = current
};

// Owns an emp_puzzle built from a piece set and an optional visiting order.
class emp_puzzle_owner {
  public:
    emp_puzzle_owner(const emp_piece_set& pieces, const emp_strategy_generator* strategy);
    ~emp_puzzle_owner();
    emp_puzzle_owner(const emp_puzzle_owner&) = delete;
    emp_puzzle_owner& operator=(const emp_puzzle_owner&) = delete;
    emp_puzzle get() const { return m_puzzle; }

  private:
    emp_puzzle m_puzzle = nullptr;
};

// Exhaustive count of all solutions in the strategy's position order (emp_strategy's
// node and solution accounting), printing the first solution's board and the totals.
class feature_CUDA_backtracker : public feature_if {
  public:
    feature_CUDA_backtracker(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                             const feature_options& options = {}, std::ostream& out = std::cout);
    void run() override;
    const emp_bt_result& get_result() const { return m_result; }

  private:
    const emp_piece_set& m_pieces;
    const emp_strategy_generator& m_strategy;
    feature_options m_options;
    std::ostream& m_out;
    emp_bt_result m_result{};
};

// The reference's solution file (include/emp_situation_binary_dumper.h:58-124):
// header, visiting order, one record per solution (the placed pieces of each level
// packed on bits(n-1)+2 bits, then the node index) and the final node count.
void write_results_bin(const std::string& path, const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                       const std::vector<emp_bt_solution>& solutions, uint64_t total_nodes);

// The exhaustive search of emp_strategy (feature new_strategy) run on the GPU: every
// solution in the reference's order, written to the dump file, and the totals.  The
// reference's "New max" progress lines belong to its sequential walk and are not printed.
class feature_new_strategy : public feature_if {
  public:
    feature_new_strategy(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                         const std::string& dump_file, const feature_options& options = {},
                         std::ostream& out = std::cout);
    void run() override;

  private:
    const emp_piece_set& m_pieces;
    const emp_strategy_generator& m_strategy;
    std::string m_dump_file;
    feature_options m_options;
    std::ostream& m_out;
};

// Greedy max-placement search, printing the final board as launch_CUDA_glutton_max does.
class feature_CUDA_glutton_max : public feature_if {
  public:
    feature_CUDA_glutton_max(const emp_piece_set& pieces, const feature_options& options = {},
                             std::ostream& out = std::cout);
    void run() override;
    const emp_gm_result& get_result() const { return m_result; }

  private:
    const emp_piece_set& m_pieces;
    feature_options m_options;
    std::ostream& m_out;
    emp_gm_result m_result{};
};

// The reference's CUDA glutton wide (include/feature_CUDA_glutton_wide.h): its launcher
// prepares the first situation of the search and prints it (src/CUDA_glutton_wide.cu:
// 27-37, CUDA_glutton_situation::print in include/CUDA_glutton_situation.h:127-156).
class feature_CUDA_glutton_wide : public feature_if {
  public:
    feature_CUDA_glutton_wide(const emp_piece_set& pieces, std::ostream& out = std::cout);
    void run() override;

  private:
    const emp_piece_set& m_pieces;
    std::ostream& m_out;
};

// One position info as the reference prints it (include/CUDA_piece_position_info2.h:
// 315-352): per non-zero word its value, the eight piece ids and their orientations.
void print_position_info(std::ostream& out, const uint32_t* words);

class factory_feature {
  public:
    // Creates the feature by name ("CUDA_backtracker", "CUDA_glutton_max",
    // "CUDA_glutton_wide", "new_strategy", "new_text_strategy").  The
    // caller owns the returned object.  Other names throw "Unsupported feature".
    static feature_if& create_feature(const std::string& feature_name, const emp_piece_set& pieces,
                                      std::unique_ptr<emp_strategy_generator>& strategy,
                                      const feature_options& options = {}, std::ostream& out = std::cout,
                                      const std::string& dump_file = "results.bin");
};

}  // namespace edge_matching_puzzle

// C++ host layer over the C ABI: features, factory, parser, strategy generators.
#include "emp_host.h"

#include <algorithm>
#include <chrono>
#include <fstream>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <sstream>

namespace edge_matching_puzzle {

namespace {

[[noreturn]] void throw_abi(const char* call, emp_status status, unsigned line)
{
    std::ostringstream s;
    s << call << " failed (status " << status << "): " << emp_last_error();
    throw emp_logic_error(s.str(), line, __FILE__);
}

std::string trim(const std::string& s)
{
    size_t b = s.find_first_not_of(" \t\r\n"), e = s.find_last_not_of(" \t\r\n");
    return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
}

}  // namespace

emp_piece_set parse_pieces(const std::string& path)
{
    std::ifstream in(path);
    if (!in) throw emp_logic_error("Unable to open file \"" + path + "\" for reading", __LINE__, __FILE__);
    std::string line;
    if (!std::getline(in, line) || trim(line) != "Width,Height")
        throw emp_logic_error("Bad header line in \"" + path + "\": expected Width,Height", __LINE__, __FILE__);
    emp_piece_set set;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "%u,%u", &set.width, &set.height) != 2)
        throw emp_logic_error("Bad dimension line in \"" + path + "\"", __LINE__, __FILE__);
    if (!std::getline(in, line) || trim(line) != "I,N,E,S,O")
        throw emp_logic_error("Bad header line in \"" + path + "\": expected I,N,E,S,O", __LINE__, __FILE__);
    const uint64_t n = static_cast<uint64_t>(set.width) * set.height;
    if (!set.width || !set.height || n > 256)
        throw emp_logic_error("Unsupported puzzle dimensions in \"" + path + "\"", __LINE__, __FILE__);
    set.colours.assign(4 * n, 0);
    std::vector<bool> seen(n, false);
    uint32_t count = 0;
    while (std::getline(in, line)) {
        if (trim(line).empty()) continue;
        unsigned id, c[4];
        if (std::sscanf(line.c_str(), "%u,%u,%u,%u,%u", &id, &c[0], &c[1], &c[2], &c[3]) != 5)
            throw emp_logic_error("Bad piece line \"" + trim(line) + "\" in \"" + path + "\"", __LINE__, __FILE__);
        if (!id || id > n || seen[id - 1])
            throw emp_logic_error("Bad piece id " + std::to_string(id) + " in \"" + path + "\"", __LINE__, __FILE__);
        seen[id - 1] = true;
        for (unsigned s = 0; s < 4; ++s) {
            if (c[s] > 255) throw emp_logic_error("Bad colour in \"" + path + "\"", __LINE__, __FILE__);
            set.colours[4 * (id - 1) + s] = static_cast<uint8_t>(c[s]);
        }
        ++count;
    }
    if (count != n) {
        std::ostringstream s;
        s << "Inconsistency between puzzle dimensions (" << set.width << "*" << set.height << ") and piece number ("
          << count << ")";
        throw emp_logic_error(s.str(), __LINE__, __FILE__);
    }
    return set;
}

namespace {

void check_order(const std::vector<uint16_t>& order, uint32_t n)
{
    std::vector<bool> used(n, false);
    for (uint16_t p : order) {
        if (p >= n || used[p]) throw emp_logic_error("The strategy does not list every position once", __LINE__, __FILE__);
        used[p] = true;
    }
}

}  // namespace

std::unique_ptr<emp_strategy_generator> create_strategy_generator(const std::string& name, uint32_t width,
                                                                  uint32_t height)
{
    const uint32_t n = width * height;
    std::vector<uint16_t> order;
    order.reserve(n);
    if (name == "basic") {
        for (uint32_t i = 0; i < n; ++i) order.push_back(static_cast<uint16_t>(i));
    } else if (name == "spiral") {
        // walk the frame inwards: right along the top, down, left, up, one ring at a time
        std::vector<bool> used(n, false);
        uint32_t x = 0, y = 0;
        for (uint32_t i = 0; i < n; ++i) {
            used[y * width + x] = true;
            order.push_back(static_cast<uint16_t>(y * width + x));
            if (i + 1 == n) break;
            if (x >= y) {
                if (x + 1 < width && !used[y * width + x + 1]) ++x;
                else if (y + 1 < height && !used[(y + 1) * width + x]) ++y;
                else --x;
            } else {
                if (x && !used[y * width + x - 1]) --x;
                else if (y && !used[(y - 1) * width + x]) --y;
                else ++x;
            }
        }
    } else {
        std::ifstream text(name);
        if (!text.is_open()) throw emp_logic_error("Unable to open file \"" + name + "\"", __LINE__, __FILE__);
        std::string line;
        for (uint32_t line_number = 1; order.size() < n && std::getline(text, line); ++line_number) {
            if (line.empty() || line[0] == '#') continue;
            const size_t comma = line.find(',');
            if (comma == std::string::npos)
                throw emp_logic_error("Missing ',' character in line " + std::to_string(line_number) + " : \"" + line +
                                          "\"", __LINE__, __FILE__);
            if (comma + 1 >= line.size())
                throw emp_logic_error("Missing information after ',' character in line " +
                                          std::to_string(line_number) + " : \"" + line + "\"", __LINE__, __FILE__);
            const long x = std::atol(line.substr(0, comma).c_str()), y = std::atol(line.substr(comma + 1).c_str());
            if (x < 0 || y < 0 || static_cast<uint32_t>(x) >= width || static_cast<uint32_t>(y) >= height)
                throw emp_logic_error("Position (" + std::to_string(x) + "," + std::to_string(y) +
                                          ") outside the puzzle in line " + std::to_string(line_number), __LINE__,
                                      __FILE__);
            order.push_back(static_cast<uint16_t>(y * width + x));
        }
        if (order.size() != n)
            throw emp_logic_error("Incomplete strategy file \"" + name + "\" : " + std::to_string(order.size()) +
                                      " < " + std::to_string(n), __LINE__, __FILE__);
        check_order(order, n);
        return std::make_unique<emp_strategy_generator>("text_generator", width, height, std::move(order));
    }
    return std::make_unique<emp_strategy_generator>(name, width, height, std::move(order));
}

std::unique_ptr<emp_strategy_generator> read_stream_strategy(std::istream& in, uint32_t width, uint32_t height)
{
    const uint32_t n = width * height;
    std::vector<uint16_t> order;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t xy[2];
        in.read(reinterpret_cast<char*>(xy), sizeof(xy));
        if (!in) throw emp_logic_error("Truncated strategy stream", __LINE__, __FILE__);
        if (xy[0] >= width || xy[1] >= height)
            throw emp_logic_error("Position outside the puzzle in strategy stream", __LINE__, __FILE__);
        order.push_back(static_cast<uint16_t>(xy[1] * width + xy[0]));
    }
    check_order(order, n);
    return std::make_unique<emp_strategy_generator>("stream_generator", width, height, std::move(order));
}

std::vector<uint16_t> situation_transitions(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                                            const std::string& situation)
{
    const uint32_t n = pieces.size();
    const size_t wd = std::to_string(n).size() + 1;
    if (situation.size() != n * wd)
        throw emp_logic_error("Situation string of " + std::to_string(situation.size()) + " characters, expected " +
                                  std::to_string(n * wd), __LINE__, __FILE__);
    // kind index of each piece: its rank among the pieces with as many frame sides
    std::vector<uint32_t> kind_index(n);
    uint32_t seen[3] = {0, 0, 0};
    for (uint32_t p = 0; p < n; ++p) {
        uint32_t zeros = 0;
        for (uint32_t s = 0; s < 4; ++s) zeros += pieces.colours[4 * p + s] == 0;
        if (zeros > 2) throw emp_logic_error("Piece with more than two frame sides", __LINE__, __FILE__);
        kind_index[p] = seen[zeros]++;
    }
    std::vector<uint16_t> out;
    for (uint16_t pos : strategy.order()) {
        const std::string cell = situation.substr(pos * wd, wd);
        if (cell.substr(0, wd - 1) == std::string(wd - 1, '-')) break;
        const char o = cell[wd - 1];
        const char* letters = "NESW";
        const char* at = std::strchr(letters, o);
        if (!o || !at) throw emp_logic_error("Bad orientation '" + std::string(1, o) + "' in situation", __LINE__, __FILE__);
        const long id = std::atol(cell.substr(0, wd - 1).c_str());
        if (id < 1 || static_cast<uint32_t>(id) > n)
            throw emp_logic_error("Bad piece id in situation: \"" + cell + "\"", __LINE__, __FILE__);
        out.push_back(static_cast<uint16_t>((kind_index[id - 1] << 2) | static_cast<uint32_t>(at - letters)));
    }
    return out;
}

std::string situation_string(uint32_t width, uint32_t height, const uint32_t* cells)
{
    const uint32_t n = width * height;
    const size_t digits = std::to_string(n).size();
    std::string out;
    out.reserve(n * (digits + 1));
    for (uint32_t pos = 0; pos < n; ++pos) {
        const uint32_t c = cells[pos];
        if (c == 0xFFFFFFFFu) {
            out.append(digits + 1, '-');
        } else {
            const std::string id = std::to_string((c >> 2) + 1);
            out.append(digits - id.size(), ' ');
            out += id;
            out += "NESW"[c & 3u];
        }
    }
    return out;
}

emp_puzzle_owner::emp_puzzle_owner(const emp_piece_set& pieces, const emp_strategy_generator* strategy)
{
    emp_puzzle_desc desc{};
    desc.width = pieces.width;
    desc.height = pieces.height;
    desc.colours = pieces.colours.data();
    desc.order = strategy ? strategy->order().data() : nullptr;
    const emp_status st = emp_puzzle_create(&desc, &m_puzzle);
    if (st != EMP_OK) throw_abi("emp_puzzle_create", st, __LINE__);
}

emp_puzzle_owner::~emp_puzzle_owner() { emp_puzzle_destroy(m_puzzle); }

feature_CUDA_backtracker::feature_CUDA_backtracker(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                                                   const feature_options& options, std::ostream& out)
    : m_pieces(pieces), m_strategy(strategy), m_options(options), m_out(out)
{
}

void feature_CUDA_backtracker::run()
{
    const auto start = std::chrono::steady_clock::now();
    emp_puzzle_owner puzzle(m_pieces, &m_strategy);
    if (m_options.trace) {
        // debug mode: the reference's own variable-space search, with the lines its
        // kernel printed for every selection (src/CUDA_backtracker.cu:109-120)
        std::vector<emp_vs_event> events(1u << 20);
        uint64_t n_events = 0;
        std::vector<uint32_t> board(m_pieces.size());
        uint32_t found = 0;
        m_out << "Launch kernels" << std::endl;
        const emp_status st = emp_bt_variable_space(puzzle.get(), m_options.device, 0, m_options.timeout_ms,
                                                    events.data(), events.size(), &n_events, board.data(), &found);
        if (st < 0) throw_abi("emp_bt_variable_space", st, __LINE__);
        for (uint64_t i = 0; i < std::min<uint64_t>(n_events, events.size()); ++i)
            m_out << "Thread " << events[i].lane << " : selected variable " << events[i].variable << " at step "
                  << events[i].step << std::endl;
        if (found) m_out << situation_string(m_pieces.width, m_pieces.height, board.data()) << std::endl;
        else m_out << "No solution" << std::endl;
        const std::chrono::duration<double> elapsed = std::chrono::steady_clock::now() - start;
        m_out << "Total elapsed time: " << elapsed.count() << "s" << std::endl;
        return;
    }
    emp_bt_config cfg{};
    cfg.device = m_options.device;
    cfg.split_depth = m_options.split_depth;
    cfg.stop_at_first = m_options.stop_at_first ? 1u : 0u;
    cfg.timeout_ms = m_options.timeout_ms;
    m_out << "Launch kernels" << std::endl;
    emp_status st;
    if (!m_options.initial_situation.empty()) {
        const std::vector<uint16_t> sit = situation_transitions(m_pieces, m_strategy, m_options.initial_situation);
        st = emp_bt_resume(puzzle.get(), sit.data(), static_cast<uint32_t>(sit.size()), &cfg, &m_result);
        if (st < 0) throw_abi("emp_bt_resume", st, __LINE__);
    } else {
        st = emp_bt_count(puzzle.get(), &cfg, &m_result);
        if (st < 0) throw_abi("emp_bt_count", st, __LINE__);
    }
    // the first solution in visiting order, as the reference's backtracker prints it
    if (m_result.has_first_solution)
        m_out << situation_string(m_pieces.width, m_pieces.height, m_result.first_solution) << std::endl;
    if (st == EMP_INCOMPLETE) m_out << "Search stopped before the end (status " << m_result.status << ")" << std::endl;
    if (st == EMP_FIRST_LOST) m_out << "First solution not recorded: " << emp_last_error() << std::endl;
    m_out << "End of algorithm" << std::endl;
    m_out << "Total situations explored : " << m_result.nodes << std::endl;
    m_out << "Nb solutions : " << m_result.solutions << std::endl;
    const std::chrono::duration<double> elapsed = std::chrono::steady_clock::now() - start;
    m_out << "Total elapsed time: " << elapsed.count() << "s" << std::endl;
}

void write_results_bin(const std::string& path, const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                       const std::vector<emp_bt_solution>& solutions, uint64_t total_nodes)
{
    std::ofstream f(path, std::ios::binary);
    if (!f) throw emp_logic_error("Unable to open file \"" + path + "\" for writing", __LINE__, __FILE__);
    const uint32_t n = pieces.size();
    auto put32 = [&](uint32_t v) { f.write(reinterpret_cast<const char*>(&v), 4); };
    auto put64 = [&](uint64_t v) { f.write(reinterpret_cast<const char*>(&v), 8); };
    put32(1);
    put32(pieces.width);
    put32(pieces.height);
    put32(1);
    for (uint32_t i = 0; i < n; ++i) {
        const auto xy = strategy.get_position(i);
        put32(xy.first);
        put32(xy.second);
    }
    uint32_t id_bits = 0;
    for (uint32_t v = n - 1; v; v >>= 1) ++id_bits;
    const uint32_t field = id_bits + 2;
    std::vector<uint64_t> words((static_cast<uint64_t>(n) * field + 63) / 64);
    for (const emp_bt_solution& s : solutions) {
        std::fill(words.begin(), words.end(), 0);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t v = s.board[strategy.order()[i]];
            for (uint32_t b = 0; b < field; ++b)
                if ((v >> b) & 1u) {
                    const uint64_t bit = static_cast<uint64_t>(i) * field + b;
                    words[bit >> 6] |= 1ull << (bit & 63);
                }
        }
        f.write(reinterpret_cast<const char*>(words.data()), static_cast<std::streamsize>(8 * words.size()));
        put64(s.node_index);
    }
    put64(total_nodes);
    if (!f) throw emp_logic_error("Write error on \"" + path + "\"", __LINE__, __FILE__);
}

feature_new_strategy::feature_new_strategy(const emp_piece_set& pieces, const emp_strategy_generator& strategy,
                                           const std::string& dump_file, const feature_options& options,
                                           std::ostream& out)
    : m_pieces(pieces), m_strategy(strategy), m_dump_file(dump_file), m_options(options), m_out(out)
{
}

void feature_new_strategy::run()
{
    emp_puzzle_owner puzzle(m_pieces, &m_strategy);
    emp_bt_config cfg{};
    cfg.device = m_options.device;
    cfg.split_depth = m_options.split_depth;
    cfg.timeout_ms = m_options.timeout_ms;
    std::vector<emp_bt_solution> sols(1024);
    uint64_t found = 0;
    emp_bt_result res{};
    // --initial_situation: emp_strategy::set_initial_state, then the search from there
    std::vector<uint16_t> sit;
    if (!m_options.initial_situation.empty())
        sit = situation_transitions(m_pieces, m_strategy, m_options.initial_situation);
    auto dump = [&]() {
        return emp_bt_resume_solutions(puzzle.get(), sit.data(), static_cast<uint32_t>(sit.size()), &cfg, sols.data(),
                                       sols.size(), &found, &res);
    };
    emp_status st = dump();
    if (st == EMP_OK && found > sols.size()) {
        sols.resize(found);
        st = dump();
    }
    if (st != EMP_OK) throw_abi("emp_bt_resume_solutions", st, __LINE__);
    sols.resize(found);
    write_results_bin(m_dump_file, m_pieces, m_strategy, sols, res.nodes);
    m_out << "End of algorithm" << std::endl;
    m_out << "Total situations explored : " << res.nodes << std::endl;
    m_out << "Nb solutions : " << res.solutions << std::endl;
}

feature_CUDA_glutton_max::feature_CUDA_glutton_max(const emp_piece_set& pieces, const feature_options& options,
                                                   std::ostream& out)
    : m_pieces(pieces), m_options(options), m_out(out)
{
}

void feature_CUDA_glutton_max::run()
{
    emp_puzzle_owner puzzle(m_pieces, nullptr);
    emp_gm_config cfg{};
    cfg.device = m_options.device;
    cfg.push_budget = m_options.push_budget;
    cfg.timeout_ms = m_options.timeout_ms;
    m_out << "Launch kernels" << std::endl;
    const emp_status st = emp_glutton_max(puzzle.get(), &cfg, &m_result);
    if (st < 0) throw_abi("emp_glutton_max", st, __LINE__);
    if (m_result.status == 2) {
        m_out << "Empty stack" << std::endl;
    } else {
        m_out << "Situation with stack played info:" << std::endl;
        m_out << situation_string(m_pieces.width, m_pieces.height, m_result.final_board) << std::endl;
    }
    m_out << "Max level : " << m_result.max_level << std::endl;
}

void print_position_info(std::ostream& out, const uint32_t* words)
{
    static const char kShort[4] = {'N', 'E', 'S', 'W'};
    for (uint32_t w = 0; w < 32; ++w) {
        uint32_t word = words[w];
        if (!word) continue;
        char hex[16];
        std::snprintf(hex, sizeof(hex), "%08x", word);
        out << "/" << std::string(8, '-') << " Word[" << std::setw(2) << w << "] : 0x" << hex << " "
            << std::string(8, '-') << "\\" << std::endl;
        for (uint32_t k = 0; k < 8; ++k) out << "|" << std::setw(4) << 8 * w + k;
        out << "|" << std::endl;
        for (uint32_t k = 0; k < 8; ++k) {
            out << "|";
            for (uint32_t o = 0; o < 4; ++o) out << (((word >> o) & 1u) ? kShort[o] : ' ');
            word >>= 4;
        }
        out << "|" << std::endl;
    }
}

feature_CUDA_glutton_wide::feature_CUDA_glutton_wide(const emp_piece_set& pieces, std::ostream& out)
    : m_pieces(pieces), m_out(out)
{
}

void feature_CUDA_glutton_wide::run()
{
    emp_puzzle_owner puzzle(m_pieces, nullptr);
    const uint32_t n = m_pieces.width * m_pieces.height;
    std::vector<uint32_t> infos(static_cast<size_t>(n) * 32);
    const emp_status st = emp_glutton_wide_situation(puzzle.get(), infos.data(), infos.size());
    if (st < 0) throw_abi("emp_glutton_wide_situation", st, __LINE__);
    // the first situation: level 0, situation index 0, info index j holds position j
    m_out << "Situation Level 0: " << std::endl;
    m_out << "Situation Index 0: " << std::endl;
    m_out << "===== Position index <-> Info index =====" << std::endl;
    for (uint32_t j = 0; j < n; ++j) m_out << "Position[" << j << "] -> Index " << j << std::endl;
    for (uint32_t j = 0; j < n; ++j) m_out << "Index[" << j << "] -> Position " << j << std::endl;
    for (uint32_t j = 0; j < n; ++j) {
        m_out << "Info[" << j << "]:" << std::endl;
        print_position_info(m_out, &infos[static_cast<size_t>(j) * 32]);
        m_out << std::endl;
    }
    for (uint32_t j = 0; j < n; ++j) {
        m_out << "Theoric info[" << j << "]:" << std::endl;
        print_position_info(m_out, &infos[static_cast<size_t>(j) * 32]);
        m_out << std::endl;
    }
    m_out << std::endl;
}

feature_if& factory_feature::create_feature(const std::string& feature_name, const emp_piece_set& pieces,
                                            std::unique_ptr<emp_strategy_generator>& strategy,
                                            const feature_options& options, std::ostream& out,
                                            const std::string& dump_file)
{
    if (feature_name == "new_strategy" || feature_name == "new_text_strategy") {
        // the reference's default orders for these features: the spiral, and the text
        // strategy file strategy.txt (src/main.cpp:103-110)
        if (!strategy)
            strategy = create_strategy_generator(feature_name == "new_strategy" ? "spiral" : "strategy.txt",
                                                 pieces.width, pieces.height);
        return *new feature_new_strategy(pieces, *strategy, dump_file, options, out);
    }
    if (feature_name == "CUDA_backtracker") {
        if (!strategy) strategy = create_strategy_generator("basic", pieces.width, pieces.height);
        return *new feature_CUDA_backtracker(pieces, *strategy, options, out);
    }
    if (feature_name == "CUDA_glutton_max") return *new feature_CUDA_glutton_max(pieces, options, out);
    if (feature_name == "CUDA_glutton_wide") return *new feature_CUDA_glutton_wide(pieces, out);
    throw emp_logic_error("Unsupported feature \"" + feature_name + "\"", __LINE__, __FILE__);
}

}  // namespace edge_matching_puzzle

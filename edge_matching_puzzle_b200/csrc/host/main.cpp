// edge_matching_puzzle: command line of the GPU features, with the reference's
// argument layout (src/main.cpp:29-146):
//
//   edge_matching_puzzle <definition.csv> <ressources> <feature_name> [--name=value ...]
//
// Feature names: CUDA_backtracker, CUDA_glutton_max, new_strategy and new_text_strategy
// (the exhaustive search with its solution file, on the GPU).  Options the reference
// takes:
//   --strategy=basic|spiral|<file>  position order (CUDA_backtracker: basic, new_strategy:
//                             spiral, new_text_strategy: the text file strategy.txt)
//   --dump_file=<path>        new_strategy's solution file (default results.bin)
//   --initial_situation=<s>   new_strategy, CUDA_backtracker: resume the search from the
//                             situation string s (emp_strategy::set_initial_state)
//   --enable_gui=...          accepted and ignored (there is no GUI here)
//   --hint                    accepted and ignored
//   --trace=true              CUDA_backtracker: run the reference's variable-space search
//                             instead and print its "Thread L : selected variable V at
//                             step S" lines (a debug mode, puzzles of at most 64 pieces)
// Settings the reference hard-codes, exposed here:
//   --stop_at_first=true|false  --split_depth=N  --push_budget=N  --timeout_ms=N  --device=N
// Errors print "ERROR : <what> at <file>:<line>" and exit with -1.
#include "emp_host.h"

#include <cstdlib>
#include <iostream>
#include <map>
#include <string>

using namespace edge_matching_puzzle;

namespace {

bool parse_bool(const std::string& v)
{
    if (v == "true" || v == "1") return true;
    if (v == "false" || v == "0") return false;
    throw emp_logic_error("Bad boolean value \"" + v + "\"", __LINE__, __FILE__);
}

uint64_t parse_u64(const std::string& name, const std::string& v)
{
    char* end = nullptr;
    const unsigned long long x = std::strtoull(v.c_str(), &end, 10);
    if (v.empty() || *end) throw emp_logic_error("Bad value \"" + v + "\" for --" + name, __LINE__, __FILE__);
    return x;
}

}  // namespace

int main(int argc, char** argv)
{
    try {
        std::vector<std::string> positional;
        std::map<std::string, std::string> named;
        for (int i = 1; i < argc; ++i) {
            const std::string a = argv[i];
            if (a.rfind("--", 0) == 0) {
                const size_t eq = a.find('=');
                if (eq == std::string::npos) throw emp_logic_error("Option " + a + " needs a value", __LINE__, __FILE__);
                named[a.substr(2, eq - 2)] = a.substr(eq + 1);
            } else {
                positional.push_back(a);
            }
        }
        if (positional.size() != 3)
            throw emp_logic_error("usage: edge_matching_puzzle <definition> <ressources> <feature_name> [--name=value]",
                                  __LINE__, __FILE__);
        static const char* known[] = {"strategy", "enable_gui", "dump_file", "initial_situation", "hint",
                                      "stop_at_first", "split_depth", "push_budget", "timeout_ms", "device",
                                      "trace"};
        for (const auto& kv : named) {
            bool ok = false;
            for (const char* k : known) ok = ok || kv.first == k;
            if (!ok) throw emp_logic_error("Unknown parameter \"" + kv.first + "\"", __LINE__, __FILE__);
        }
        feature_options options;
        if (named.count("stop_at_first")) options.stop_at_first = parse_bool(named["stop_at_first"]);
        if (named.count("enable_gui")) parse_bool(named["enable_gui"]);
        if (named.count("split_depth"))
            options.split_depth = static_cast<uint32_t>(parse_u64("split_depth", named["split_depth"]));
        if (named.count("push_budget")) options.push_budget = parse_u64("push_budget", named["push_budget"]);
        if (named.count("timeout_ms"))
            options.timeout_ms = static_cast<uint32_t>(parse_u64("timeout_ms", named["timeout_ms"]));
        if (named.count("device")) options.device = static_cast<int>(parse_u64("device", named["device"]));
        if (named.count("initial_situation")) options.initial_situation = named["initial_situation"];
        if (named.count("trace")) options.trace = parse_bool(named["trace"]);

        const emp_piece_set pieces = parse_pieces(positional[0]);
        std::cout << pieces.size() << " pieces loaded" << std::endl;
        std::unique_ptr<emp_strategy_generator> strategy;
        if (named.count("strategy"))
            strategy = create_strategy_generator(named["strategy"], pieces.width, pieces.height);
        const std::string dump_file = named.count("dump_file") ? named["dump_file"] : "results.bin";
        std::unique_ptr<feature_if> feature(
            &factory_feature::create_feature(positional[2], pieces, strategy, options, std::cout, dump_file));
        feature->run();
    } catch (emp_logic_error& e) {
        std::cout << "ERROR : " << e.what() << " at " << e.get_file() << ":" << e.get_line() << std::endl;
        return -1;
    }
    return 0;
}

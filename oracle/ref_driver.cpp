// Command-line driver around the reference's own new_strategy search
// (include/emp_strategy.h), compiled unmodified from the reference sources with
// the project-written stand-ins of oracle/ref_shim/ for its external libraries.
// Test infrastructure only: it pins oracle/emp_oracle.c (and through it the CUDA
// path) on the reference itself.  Nothing in the library links or runs it.
//
// It follows the reference's main for the new_strategy feature
// (src/main.cpp:55-133 and include/factory_feature.h:133-140): parse the puzzle
// file, build emp_piece_db and emp_FSM_info, create the position-order generator
// (basic, spiral or a text strategy file) and run emp_strategy, optionally after
// set_initial_state (the --initial_situation parameter).  The reference prints
// its own lines ("New max : L", "Total situations explored : N", "Nb solutions :
// S") and writes results.bin; this driver adds one line with the number of
// identical-mask writes that fell outside a bitfield (see quicky_bitfield.h).
//
//   emp_ref_strategy <puzzle file> [strategy] [dump file] [initial situation]
//     strategy: basic (default), spiral or a text strategy file name
#include "emp_FSM_info.h"
#include "emp_FSM_situation.h"
#include "emp_gui.h"
#include "emp_piece_db.h"
#include "emp_pieces_parser.h"
#include "emp_strategy.h"
#include "emp_strategy_generator_factory.h"

#include <iostream>
#include <memory>
#include <string>
#include <vector>

using namespace edge_matching_puzzle;

// set_initial_state ends with sleep(20) (include/emp_strategy.h:464), a pause for
// its GUI; the build maps sleep to this no-op.
extern "C" unsigned int ref_shim_sleep(unsigned int) { return 0; }

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " <puzzle file> [basic|spiral|strategy file] [dump file] [initial situation]"
                  << std::endl;
        return 2;
    }
    const std::string strategy = argc > 2 ? argv[2] : "basic";
    const std::string dump = argc > 3 && std::string(argv[3]).size() ? argv[3] : "/dev/null";
    const std::string initial = argc > 4 ? argv[4] : "";
    try {
        std::vector<emp_piece> pieces;
        emp_pieces_parser parser(argv[1]);
        unsigned int width = 0, height = 0;
        parser.parse(width, height, pieces);
        std::cout << pieces.size() << " pieces loaded" << std::endl;
        emp_gui gui;
        emp_piece_db piece_db(pieces, width, height);
        emp_FSM_info info(width, height, piece_db.get_piece_id_size(), piece_db.get_dumped_piece_id_size());
        emp_FSM_situation::init(info);
        std::unique_ptr<emp_strategy_generator> generator(emp_strategy_generator_factory::create(strategy, info));
        generator->generate();
        std::cout << "identical-mask writes outside a bitfield : " << quicky_utils::bitfield_out_of_range_counter()
                  << std::endl;
        emp_strategy search(generator, piece_db, gui, info, dump);
        if (!initial.empty()) search.set_initial_state(initial);
        search.run();
    } catch (quicky_exception::quicky_runtime_exception& e) {
        std::cout << "ERROR : " << e.what() << " at " << e.get_file() << ":" << e.get_line() << std::endl;
        return -1;
    } catch (quicky_exception::quicky_logic_exception& e) {
        std::cout << "ERROR : " << e.what() << " at " << e.get_file() << ":" << e.get_line() << std::endl;
        return -1;
    }
    return 0;
}

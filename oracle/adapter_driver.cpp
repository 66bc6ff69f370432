// Test infrastructure: drives the B200 engine through the reference's own
// algorithm interface, the way ExperimentManager::perform_alg does
// (src/infrastructure/experiment_manager.hpp:365-394): set_params, then the
// five phases wrapped in the reference's TimedAlgorithm (algorithm.hpp:220-280)
// so each phase is timed by its Timer, then validation against the
// reference's default validator GoLCpuNaive<char> with Grid::equals
// (experiment_manager.hpp:272-307, experiment_params.hpp:43).
//
// Built by `make -C oracle adapter` from the reference sources in place, into
// oracle/_ref/adapter_driver. Usage:
//   adapter_driver X Y ITERATIONS SEED [temporal_steps] [local|k1|resident]
// `k1` registers the adapter with its depth forced to one generation per
// pass (GolB200Algorithm<char, GOL_ALG_AUTO, 1>) and checks that the engine
// ran at that depth.
// Exit status 0 iff the engine's grid equals the reference's.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "algorithms/cpu-naive/gol_cpu_naive.hpp"
#include "gol_b200_algorithm.hpp"
#include "infrastructure/algorithm.hpp"
#include "infrastructure/data_loader.hpp"

template <typename Alg>
static infrastructure::Grid<2, char> perform(Alg& alg, const infrastructure::ExperimentParams& p,
                                             const infrastructure::Grid<2, char>& input,
                                             bool timed) {
    alg.set_params(p);
    if (timed) {
        infrastructure::TimedAlgorithm<2, char> t(&alg);
        t.set_params(p);
        t.set_and_format_input_data(input);
        t.initialize_data_structures();
        t.run(p.iterations);
        t.finalize_data_structures();
        auto out = t.fetch_result();
        std::printf("%s", t.get_time_report().pretty_print().c_str());
        return out;
    }
    alg.set_and_format_input_data(input);
    alg.initialize_data_structures();
    alg.run(p.iterations);
    alg.finalize_data_structures();
    return alg.fetch_result();
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s X Y ITERATIONS SEED [temporal_steps] [local|k1|resident]\n", argv[0]);
        return 2;
    }
    infrastructure::ExperimentParams p;
    p.grid_dimensions = {std::strtoull(argv[1], nullptr, 10), std::strtoull(argv[2], nullptr, 10)};
    p.iterations = std::strtoull(argv[3], nullptr, 10);
    p.random_seed = std::strtoull(argv[4], nullptr, 10);
    p.temporal_steps = argc > 5 ? std::strtoull(argv[5], nullptr, 10) : 1;
    p.state_bits_count = 64;
    p.max_runtime_seconds = infrastructure::StopWatch::MAX_TIME;
    p.animate_output = false;
    c::set_colorful(false);

    infrastructure::RandomOnesZerosDataLoader<2, char> loader;
    auto input = loader.load_data(p);

    infrastructure::Grid<2, char> got;
    try {
        if (argc > 6 && std::strcmp(argv[6], "local") == 0) {
            golb200::GolB200Algorithm<char, GOL_ALG_LOCAL> alg;
            for (int round = 0; round < 2; ++round) got = perform(alg, p, input, round == 1);
        } else if (argc > 6 && std::strcmp(argv[6], "k1") == 0) {
            golb200::GolB200Algorithm<char, GOL_ALG_AUTO, 1> alg;
            for (int round = 0; round < 2; ++round) {
                got = perform(alg, p, input, round == 1);
                // gol_plan reports the depth of an initialised engine: run one
                // more generation-free round to read it back
                alg.set_and_format_input_data(input);
                alg.initialize_data_structures();
                uint32_t depth = 0;
                if (gol_plan(alg.engine(), &depth, nullptr, nullptr) != GOL_OK || depth != 1) {
                    std::fprintf(stderr, "engine depth %u, expected 1\n", depth);
                    return 4;
                }
                alg.finalize_data_structures();
                std::printf("engine depth: %u generation per pass\n", depth);
            }
        } else if (argc > 6 && std::strcmp(argv[6], "resident") == 0) {
            golb200::GolB200Algorithm<char, GOL_ALG_RESIDENT> alg;
            for (int round = 0; round < 2; ++round) got = perform(alg, p, input, round == 1);
        } else {
            golb200::GolB200Algorithm<char> alg;
            for (int round = 0; round < 2; ++round) got = perform(alg, p, input, round == 1);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "engine error: %s\n", e.what());
        return 3;
    }
    algorithms::GoLCpuNaive<char> validator;
    auto want = perform(validator, p, input, false);
    const bool ok = got.equals(want);
    std::printf("%llux%llu, %llu generations: %s\n", (unsigned long long)p.grid_dimensions[0],
                (unsigned long long)p.grid_dimensions[1], (unsigned long long)p.iterations,
                ok ? "valid (equals GoLCpuNaive)" : "INVALID");
    return ok ? 0 : 1;
}

// C++ adapter: the B200 engine behind the reference's algorithm contract.
//
// GolB200Algorithm<cell_t> derives from infrastructure::Algorithm<2, cell_t>
// (src/infrastructure/algorithm.hpp:17-87) and forwards every phase to the
// C ABI in include/gol_b200.h, so ExperimentManager can register it like any
// other algorithm (experiment_manager.hpp:80-222) and drive it through
// perform_alg (:365-394). A non-zero status from the library is thrown as
// std::runtime_error, the reference's error convention for bad shapes and
// failures (general_bit_grid.hpp:207-215, cuch.hpp:42-52).
//
// This header is compiled inside the reference's source tree: it includes the
// reference's own headers (infrastructure/algorithm.hpp) and needs
// include/gol_b200.h and libgolb200.so from this repository.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "gol_b200.h"
#include "infrastructure/algorithm.hpp"

namespace golb200 {

// Depth: 0 takes ExperimentParams::temporal_steps (whose default, 1, and 0
// let the engine pick its depth: the reference's default of one generation
// per step would be the slowest choice here); 1..16 forces that depth, so
// registering GolB200Algorithm<char, GOL_ALG_AUTO, 1> gives the
// one-generation (HBM-streaming) kernel under its own algorithm name.
template <typename cell_t, uint32_t Algo = GOL_ALG_AUTO, uint32_t Depth = 0>
class GolB200Algorithm : public infrastructure::Algorithm<2, cell_t> {
    static_assert(Depth <= 16, "depth is 1..16, or 0 for the parameters' choice");
  public:
    using DataGrid = infrastructure::Grid<2, cell_t>;
    using size_type = std::size_t;

    ~GolB200Algorithm() override { gol_destroy(engine_); }

    // set_params may be called before every round (experiment_manager.hpp:371):
    // the engine is rebuilt only when the grid or a tuning field changes.
    void set_params(const infrastructure::ExperimentParams& params) override {
        this->params = params;
    }

    void set_and_format_input_data(const DataGrid& data) override {
        x_ = data.template size_in<0>();
        y_ = data.template size_in<1>();
        ensure_engine();
        if constexpr (std::is_same_v<cell_t, std::int32_t>) {
            check(gol_set_input_i32(engine_, data.data(), x_, y_), "set_and_format_input_data");
        } else {
            static_assert(sizeof(cell_t) == 1, "cell type must be char or int32_t");
            check(gol_set_input_u8(engine_, reinterpret_cast<const uint8_t*>(data.data()), x_, y_),
                  "set_and_format_input_data");
        }
    }

    void initialize_data_structures() override { check(gol_init(engine_), "initialize_data_structures"); }

    void run(size_type iterations) override { check(gol_run(engine_, iterations), "run"); }

    void finalize_data_structures() override { check(gol_finalize(engine_), "finalize_data_structures"); }

    DataGrid fetch_result() override {
        DataGrid out(x_, y_);
        if constexpr (std::is_same_v<cell_t, std::int32_t>) {
            check(gol_fetch_i32(engine_, out.data()), "fetch_result");
        } else {
            check(gol_fetch_u8(engine_, reinterpret_cast<uint8_t*>(out.data())), "fetch_result");
        }
        return out;
    }

    std::size_t actually_performed_iterations() const override { return gol_performed(engine_); }

    // The engine behind the adapter (for gol_plan, gol_local_stats and the
    // like); null before the first set_and_format_input_data.
    gol_engine* engine() const { return engine_; }

  private:
    void ensure_engine() {
        gol_config cfg;
        gol_config_init(&cfg, x_, y_);
        cfg.algorithm = Algo;
        cfg.word_bits = this->params.state_bits_count == 32 ? 32 : 64;
        cfg.temporal_steps =
            Depth ? Depth : (this->params.temporal_steps > 1 ? (uint32_t)this->params.temporal_steps : 0);
        // ExperimentParams::thread_block_size is a CUDA block size in threads
        // for the reference's kernels; the row-band kernels size their CTAs
        // from the grid's width, so it is not passed on (band height: auto).
        cfg.thread_block_size = 0;
        cfg.max_runtime_seconds =
            this->params.max_runtime_seconds == (std::size_t)infrastructure::StopWatch::MAX_TIME
                ? 0
                : this->params.max_runtime_seconds;
        if (engine_ && same_config(cfg)) return;
        gol_destroy(engine_);
        engine_ = nullptr;
        check(gol_create(&engine_, &cfg), "gol_create");
        cfg_ = cfg;
    }

    bool same_config(const gol_config& c) const {
        return c.x == cfg_.x && c.y == cfg_.y && c.algorithm == cfg_.algorithm &&
               c.word_bits == cfg_.word_bits && c.temporal_steps == cfg_.temporal_steps &&
               c.max_runtime_seconds == cfg_.max_runtime_seconds;
    }

    void check(int rc, const char* phase) const {
        if (rc != GOL_OK)
            throw std::runtime_error(std::string("gol-b200 ") + phase + ": " + gol_last_error(engine_));
    }

    gol_engine* engine_ = nullptr;
    gol_config cfg_{};
    std::size_t x_ = 0, y_ = 0;
};

} // namespace golb200

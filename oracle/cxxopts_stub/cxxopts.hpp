// Test infrastructure (oracle build only): a minimal stand-in for the
// cxxopts option parser (jarro2783/cxxopts @ 3bf2684, fetched by the
// reference's CMake over the network, which this machine does not have).
//
// It declares just enough of the cxxopts API for the reference header
// src/infrastructure/experiment_params.hpp:152-314 to compile unmodified.
// The oracle harness never calls ParamsParser::parse, so none of these
// members do real work; parse() throws if it is ever reached.
#ifndef GOL_ORACLE_CXXOPTS_STUB_HPP
#define GOL_ORACLE_CXXOPTS_STUB_HPP

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>

namespace cxxopts {

class Value : public std::enable_shared_from_this<Value> {
  public:
    virtual ~Value() = default;
    std::shared_ptr<Value> default_value(const std::string&) { return shared_from_this(); }
};

template <typename T>
std::shared_ptr<Value> value() {
    return std::make_shared<Value>();
}

class OptionAdder {
  public:
    OptionAdder& operator()(const std::string&, const std::string&,
                            std::shared_ptr<Value> = nullptr) {
        return *this;
    }
};

class OptionValue {
  public:
    template <typename T>
    const T& as() const {
        throw std::logic_error("cxxopts stub: option values are not available");
    }
};

class ParseResult {
  public:
    std::size_t count(const std::string&) const { return 0; }
    const OptionValue& operator[](const std::string&) const { return value_; }

  private:
    OptionValue value_;
};

class Options {
  public:
    Options(std::string, std::string = "") {}
    OptionAdder add_options(std::string = "") { return OptionAdder(); }
    ParseResult parse(int, const char* const*) {
        throw std::logic_error("cxxopts stub: command-line parsing is not available");
    }
    std::string help() const { return ""; }
};

} // namespace cxxopts

#endif

#pragma once

// Free-form MPS reader (VIKALP include/vikalp/io/MpsReader.hpp, same class
// and members): NAME, ROWS (N / L / G / E), COLUMNS and RHS with one or two
// entries per line, BOUNDS (LO / UP / FX / FR / BV), ENDATA. Variables are
// numbered in order of first appearance in COLUMNS and default to [0, +inf);
// a repeated (row, variable) or objective entry keeps its last value. Every
// problem found is recorded with its line (0 for problems found after the
// file was read), in the reference's order and wording; read() returns false
// when there is any, or when the model fails Model::validate().

#include "vikalp/contracts/Model.hpp"

#include <cstddef>
#include <string>
#include <vector>

namespace vikalp {

struct MpsError {
    std::size_t line = 0;
    std::string message;
};

class MpsReader {
public:
    bool read(const std::string &path, Model &model);
    [[nodiscard]] const std::vector<MpsError> &errors() const noexcept;

private:
    std::vector<MpsError> errors_;
};

} // namespace vikalp

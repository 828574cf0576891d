// Initial conditions of the solvers (reference: src/Domains/Field/InitialConditions.h).
// case/initialConditions.info gives, per field ("u", "p"), a type and its values: uniform,
// sphere (value inside a sphere) or box (value inside an axis-aligned box).  The solver
// applies them to its device fields at construction.
#pragma once
#include <string>
#include <vector>

#include "HexaFvmMesh.h"
#include "Input.h"

class InitialConditions {
public:
    explicit InitialConditions(const Input& input) : ic_(input.initialConditions) {}
    // per-cell values of one field (components planes of nCells each), from the cell centroids
    std::vector<double> values(const std::string& field, int components, const std::vector<double>& centroids) const;
    bool has(const std::string& field) const { return ic_.has(field + ".type"); }

private:
    InfoTree ic_;
};

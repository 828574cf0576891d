// Initial conditions of the solvers (reference: src/Domains/Field/InitialConditions.h).
// case/initialConditions.info gives, per field ("u", "p"), a type and its values: uniform,
// box (value inside an axis-aligned box) or restart (the values of a restart file).  The
// reference's sphere type is rejected (its smoothing loop does not terminate).  The solver
// applies them to its device fields at construction.
//
// Restart files keep the layout of the reference's writeRestart
// (src/Domains/Field/InitialConditions.cpp:77-119): cells in i-fastest order, one text line
// per j row, an empty line after each k plane, and for a vector field the three components of
// a cell side by side.  The reference declares a reader (setFromRestart,
// InitialConditions.h:69) but never defines it; the restart type here is that reader.
#pragma once
#include <string>
#include <vector>

#include "HexaFvmMesh.h"
#include "Input.h"

class Solver;

class InitialConditions {
public:
    explicit InitialConditions(const Input& input) : ic_(input.initialConditions) {}
    // per-cell values of one field (components planes of nCells each), from the cell centroids
    std::vector<double> values(const std::string& field, int components, const std::vector<double>& centroids) const;
    bool has(const std::string& field) const { return ic_.has(field + ".type"); }

    // writes the solver's field ("u" or "p") to <field>Restart.rst in the working directory,
    // where the reference's writeRestart puts it
    void writeRestart(const Solver& solver, const std::string& field) const;

    // a field given as component planes of nI*nJ*nK cells, in the restart layout, with 17
    // significant digits so that reading it back gives the same doubles
    static void writeRestartFile(const std::string& path, const std::vector<double>& planes, int components, int nI, int nJ,
                                 int nK);
    // the component planes of a restart file of nCells cells; files written by the reference
    // (6 significant digits) read the same way
    static std::vector<double> readRestartFile(const std::string& path, int components, size_t nCells);

private:
    InfoTree ic_;
};

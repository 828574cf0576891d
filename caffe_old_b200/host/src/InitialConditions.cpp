// Initial conditions (reference: src/Domains/Field/InitialConditions.cpp/.tpp): uniform and
// box fields are evaluated at the cell centroids; restart fields are read from a restart
// file.  The reference's sphere form smooths the field with a loop whose innermost index
// never advances (InitialConditions.tpp, smootheField: `i < endI; ++ii`), so it does not
// terminate there; it is reported as unsupported instead of being given a different meaning
// here.
#include "InitialConditions.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "Output.h"
#include "Solver.h"

std::vector<double> InitialConditions::values(const std::string& field, int components, const std::vector<double>& centroids) const {
    const size_t N = centroids.size() / 3;
    std::vector<double> out((size_t)components * N, 0.);
    const std::string type = ic_.get<std::string>(field + ".type");
    auto value = [&](const std::string& key) {
        Vector3D v;
        if (components == 1) v.x = ic_.get<double>(field + "." + key);
        else v = std::stov(ic_.get<std::string>(field + "." + key));
        return v;
    };
    if (type == "uniform") {
        Vector3D v = value("value");
        for (int c = 0; c < components; ++c)
            for (size_t q = 0; q < N; ++q) out[c * N + q] = v(c);
    } else if (type == "box") {
        // the reference passes yLength for the z extent as well (InitialConditions.cpp:30-34)
        double lx = ic_.get<double>(field + ".xLength"), ly = ic_.get<double>(field + ".yLength"), lz = ly;
        Vector3D ctr = std::stov(ic_.get<std::string>(field + ".center"));
        Vector3D v = value("value");
        for (size_t q = 0; q < N; ++q) {
            double x = centroids[q], y = centroids[N + q], z = centroids[2 * N + q];
            bool in = x >= ctr.x - 0.5 * lx && x <= ctr.x + 0.5 * lx && y >= ctr.y - 0.5 * ly && y <= ctr.y + 0.5 * ly &&
                      z >= ctr.z - 0.5 * lz && z <= ctr.z + 0.5 * lz;
            if (in)
                for (int c = 0; c < components; ++c) out[c * N + q] = v(c);
        }
    } else if (type == "restart") {
        out = readRestartFile(ic_.get<std::string>(field + ".file", field + "Restart.rst"), components, N);
    } else {
        Output::raiseException("InitialConditions", "values", "initial condition type \"" + type + "\" of field \"" + field +
                                                                  "\" is not supported (uniform, box and restart are)");
    }
    return out;
}

void InitialConditions::writeRestart(const Solver& solver, const std::string& field) const {
    const HexaFvmMesh& mesh = solver.mesh();
    const std::vector<double> planes = solver.field(field);
    const size_t N = (size_t)mesh.nCells();
    if (N == 0 || planes.size() % N != 0)
        Output::raiseException("InitialConditions", "writeRestart", "field \"" + field + "\" is not a cell field");
    writeRestartFile(field + "Restart.rst", planes, (int)(planes.size() / N), mesh.nCellsI(), mesh.nCellsJ(), mesh.nCellsK());
}

void InitialConditions::writeRestartFile(const std::string& path, const std::vector<double>& planes, int components, int nI, int nJ,
                                         int nK) {
    const size_t N = (size_t)nI * nJ * nK;
    if (components < 1 || planes.size() != (size_t)components * N)
        Output::raiseException("InitialConditions", "writeRestartFile", "the field does not hold " + std::to_string(components) +
                                                                            " planes of " + std::to_string(N) + " cells");
    std::FILE* f = std::fopen(path.c_str(), "w");
    if (!f) Output::raiseException("InitialConditions", "writeRestartFile", "cannot write \"" + path + "\"");
    size_t c = 0;
    bool ok = true;
    for (int k = 0; k < nK && ok; ++k) {
        for (int j = 0; j < nJ && ok; ++j) {
            for (int i = 0; i < nI; ++i, ++c)
                for (int q = 0; q < components; ++q) ok = ok && std::fprintf(f, "%.17g ", planes[q * N + c]) > 0;
            ok = ok && std::fputc('\n', f) != EOF;
        }
        ok = ok && std::fputc('\n', f) != EOF;
    }
    ok = std::fclose(f) == 0 && ok;
    if (!ok) Output::raiseException("InitialConditions", "writeRestartFile", "writing \"" + path + "\" failed");
}

std::vector<double> InitialConditions::readRestartFile(const std::string& path, int components, size_t nCells) {
    std::ifstream f(path);
    if (!f) Output::raiseException("InitialConditions", "readRestartFile", "cannot open restart file \"" + path + "\"");
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    const size_t want = (size_t)components * nCells;
    std::vector<double> out(want, 0.);
    const char* s = text.c_str();
    size_t n = 0;
    for (;;) {
        while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r') ++s;
        if (!*s) break;
        char* end = nullptr;
        double v = std::strtod(s, &end);
        if (end == s)
            Output::raiseException("InitialConditions", "readRestartFile", "\"" + path + "\" holds a value that is not a number after " +
                                                                               std::to_string(n) + " values");
        if (n < want) out[(n % components) * nCells + n / components] = v;
        ++n;
        s = end;
    }
    if (n != want)
        Output::raiseException("InitialConditions", "readRestartFile", "\"" + path + "\" holds " + std::to_string(n) + " values; " +
                                                                           std::to_string(want) + " (" + std::to_string(components) +
                                                                           " per cell) were expected");
    return out;
}

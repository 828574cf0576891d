// Initial conditions (reference: src/Domains/Field/InitialConditions.cpp/.tpp): uniform and
// box fields are evaluated at the cell centroids.  The reference's sphere form smooths the
// field with a loop whose innermost index never advances (InitialConditions.tpp,
// smootheField: `i < endI; ++ii`), so it does not terminate there; it is reported as
// unsupported instead of being given a different meaning here.
#include "InitialConditions.h"

#include "Output.h"

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
    } else {
        Output::raiseException("InitialConditions", "values", "initial condition type \"" + type + "\" of field \"" + field +
                                                                  "\" is not supported (uniform and box are)");
    }
    return out;
}

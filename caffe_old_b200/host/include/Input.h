// Case input (reference: src/RunControl/Input.h).  The reference reads case/case.info and
// case/initialConditions.info with boost::property_tree's INFO parser; InfoTree parses the
// same format (key value lines, nested { } blocks, ';' comments, quoted strings) and offers
// the get<T>("A.B.c") lookups the solvers use.
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "Output.h"

class InfoTree {
public:
    std::string data;
    std::vector<std::pair<std::string, InfoTree>> children;

    static InfoTree readFile(const std::string& filename);
    static InfoTree parse(const std::string& text);
    const InfoTree* find(const std::string& path) const;
    bool has(const std::string& path) const { return find(path) != nullptr; }
    std::string getString(const std::string& path) const;

    template <class T>
    T get(const std::string& path) const;
    template <class T>
    T get(const std::string& path, const T& fallback) const {
        return has(path) ? get<T>(path) : fallback;
    }
};

template <>
std::string InfoTree::get<std::string>(const std::string& path) const;
template <>
double InfoTree::get<double>(const std::string& path) const;
template <>
int InfoTree::get<int>(const std::string& path) const;

class Input {
public:
    Input();
    Input(const std::string& caseFilename, const std::string& initialConditionsFilename);

    InfoTree caseParameters;
    InfoTree initialConditions;
};

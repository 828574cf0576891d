// Process layout (reference: src/Parallel/Parallel.h).  One process drives one GPU and owns
// the whole lattice: there is no domain decomposition, so every collective is the identity.
#pragma once
#include <utility>

class Parallel {
public:
    static void initialize() {}
    static void finalize() {}
    static int nProcesses() { return 1; }
    static int processNo() { return 0; }
    static int mainProcNo() { return 0; }
    static bool isMainProcessor() { return true; }
    static std::pair<int, int> ownershipRange(int nEntities) { return {0, nEntities}; }
    static double sum(double v) { return v; }
    static int sum(int v) { return v; }
    static double max(double v) { return v; }
    static double min(double v) { return v; }
    static void barrier() {}
};

// hexaMesh: generates mesh/structuredMesh.dat from mesh/structuredMesh.info (the reference's
// Modules/hexaMesh.cpp flow).
#include <iostream>

#include "HexaMeshGen.h"
#include "Output.h"
#include "Parallel.h"

int main(int argc, const char* argv[]) {
    (void)argc; (void)argv;
    Parallel::initialize();
    int rc = 0;
    try {
        HexaMeshGen gen;
        gen.readFile("mesh/");
        gen.generateMesh();
        gen.checkMesh();
        gen.writeMeshFile("mesh/");
    } catch (const char* errorMessage) {
        std::cerr << "Error: " << errorMessage << std::endl;
        rc = 1;
    }
    Parallel::finalize();
    return rc;
}

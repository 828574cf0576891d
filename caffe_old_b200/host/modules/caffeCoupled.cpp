// caffeCoupled: coupled momentum / continuity run of the case in the working directory
// (case/case.info, mesh/structuredMesh.dat), written to solution/ every
// RunControl.fileWriteInterval iterations and at the end.  Same flow as the reference's
// Modules/caffeCoupled.cpp.
#include <iostream>

#include "Coupled.h"
#include "Input.h"
#include "Parallel.h"
#include "RunControl.h"

int main(int argc, const char* argv[]) {
    (void)argc; (void)argv;
    Parallel::initialize();
    int rc = 0;
    try {
        Input input;
        RunControl runControl;
        HexaFvmMesh mesh;
        runControl.initialize(input);
        mesh.initialize("mesh/structuredMesh.dat");
        Output::print(mesh.meshStats());
        Coupled coupled(input, mesh);
        runControl.displayStartMessage();
        while (runControl.continueRun()) {
            runControl.residualNorm = coupled.solve(runControl.timeStep());
            coupled.displayUpdateMessage();
            runControl.displayUpdateMessage();
            if (runControl.writeToFile()) mesh.writeTec360(runControl.simTime(), "solution/");
        }
        runControl.displayEndMessage();
        mesh.writeTec360(runControl.simTime(), "solution/");
    } catch (const char* errorMessage) {
        std::cerr << "Error: " << errorMessage << std::endl;
        rc = 1;
    }
    Parallel::finalize();
    return rc;
}

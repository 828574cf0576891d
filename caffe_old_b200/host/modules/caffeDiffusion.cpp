// caffeDiffusion: scalar diffusion run of the case in the working directory (case/case.info,
// case/initialConditions.info, mesh/structuredMesh.dat), written to solution/ every
// RunControl.fileWriteInterval iterations and at the end.  Same flow as the reference's
// Modules/caffeDiffusion.cpp.
#include <iostream>
#include <memory>

#include "Diffusion.h"
#include "Input.h"
#include "Parallel.h"
#include "ParallelHexaFvmMesh.h"
#include "RunControl.h"

int main(int argc, const char* argv[]) {
    (void)argc; (void)argv;
    Parallel::initialize();
    std::unique_ptr<HexaFvmMesh> mesh(Parallel::nProcesses() == 1 ? new HexaFvmMesh : new ParallelHexaFvmMesh);
    int rc = 0;
    try {
        Input input;
        RunControl runControl;
        runControl.initialize(input);
        mesh->initialize("mesh/structuredMesh.dat");
        Output::print(mesh->meshStats());
        Diffusion diffusion(input, *mesh);
        runControl.displayStartMessage();
        while (runControl.continueRun()) {
            runControl.residualNorm = diffusion.solve(runControl.timeStep());
            diffusion.displayUpdateMessage();
            runControl.displayUpdateMessage();
            if (runControl.writeToFile()) mesh->writeTec360(runControl.simTime(), "solution/");
        }
        runControl.displayEndMessage();
        mesh->writeTec360(runControl.simTime(), "solution/");
    } catch (const char* errorMessage) {
        std::cerr << "Error: " << errorMessage << std::endl;
        rc = 1;
    }
    Parallel::finalize();
    return rc;
}

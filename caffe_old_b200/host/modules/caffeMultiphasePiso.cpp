// caffeMultiphasePiso: transient MultiphasePiso run of the case in the working directory (case/case.info,
// case/initialConditions.info, mesh/structuredMesh.dat), written to solution/ every
// RunControl.fileWriteInterval steps; RunControl.writeRestart ON (optional) also writes restart
// files of u and p at the end.  Same flow as the reference's Modules/caffeMultiphasePiso.cpp.
#include <iostream>
#include <memory>

#include "InitialConditions.h"
#include "Input.h"
#include "Parallel.h"
#include "ParallelHexaFvmMesh.h"
#include "MultiphasePiso.h"
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
        MultiphasePiso piso(input, *mesh);
        runControl.displayStartMessage();
        while (runControl.continueRun()) {
            runControl.residualNorm = piso.solve(runControl.timeStep());
            piso.displayUpdateMessage();
            runControl.displayUpdateMessage();
            if (runControl.writeToFile()) mesh->writeTec360(runControl.simTime(), "solution/");
        }
        runControl.displayEndMessage();
        mesh->writeTec360(runControl.simTime(), "solution/");
        // optional: uRestart.rst and pRestart.rst for a later run's restart initial conditions
        if (input.caseParameters.get<std::string>("RunControl.writeRestart", std::string("OFF")) == "ON") {
            InitialConditions ics(input);
            ics.writeRestart(piso, "u");
            ics.writeRestart(piso, "p");
        }
    } catch (const char* errorMessage) {
        std::cerr << "Error: " << errorMessage << std::endl;
        rc = 1;
    }
    Parallel::finalize();
    return rc;
}

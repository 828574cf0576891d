// Outer loop control of the module mains (reference: src/RunControl/RunControl.h):
// termination on iterations or simulated time, the time step, and the file-write interval.
#pragma once
#include <chrono>
#include <string>

#include "Input.h"

class RunControl {
public:
    RunControl();
    void initialize(const Input& input);
    bool continueRun();
    bool writeToFile() const { return itrs_ % fileWriteInterval_ == 0; }
    double timeStep() const { return timeStep_; }
    double simTime() const { return simTime_; }
    int iteration() const { return itrs_; }
    void displayStartMessage();
    void displayUpdateMessage();
    void displayEndMessage();

    double residualNorm = 0.;

private:
    int itrs_ = 0, maxIters_ = 0, fileWriteInterval_ = 1;
    double simTime_ = 0., timeStep_ = 0., maxSimTime_ = 0.;
    std::string terminationCondition_ = "iterations";
    std::chrono::steady_clock::time_point start_;
};

// Outer loop control (reference: src/RunControl/RunControl.cpp): the RunControl section of
// case/case.info; the solution/ directory for the output files.
#include "RunControl.h"

#include <sys/stat.h>

#include <cerrno>
#include <sstream>

RunControl::RunControl() = default;

void RunControl::initialize(const Input& input) {
    const InfoTree& c = input.caseParameters;
    terminationCondition_ = c.get<std::string>("RunControl.terminationCondition");
    maxIters_ = c.get<int>("RunControl.maxNumberOfIterations");
    timeStep_ = c.get<double>("RunControl.timeStep");
    maxSimTime_ = c.get<double>("RunControl.maxSimTime");
    fileWriteInterval_ = c.get<int>("RunControl.fileWriteInterval");
    if (fileWriteInterval_ < 1) fileWriteInterval_ = 1;
    if (mkdir("solution", 0755) != 0 && errno != EEXIST)
        Output::raiseException("RunControl", "initialize", "creation of directory \"solution\" failed");
    start_ = std::chrono::steady_clock::now();
}

bool RunControl::continueRun() {
    ++itrs_;
    simTime_ += timeStep_;
    if (terminationCondition_ == "iterations") return itrs_ < maxIters_;
    if (terminationCondition_ == "simTime") return simTime_ < maxSimTime_;
    if (terminationCondition_ == "realTime") {
        Output::issueWarning("RunControl", "continueRun", "termination condition for real time not yet implemented.");
        return true;
    }
    Output::raiseException("RunControl", "continueRun", "invalid termination condition \"" + terminationCondition_ + "\" selected.");
    return false;
}

void RunControl::displayStartMessage() {
    Output::print("RunControl", "Beginning simulation. Terminating on condition: " + terminationCondition_);
}

void RunControl::displayUpdateMessage() {
    double pct = terminationCondition_ == "simTime" ? simTime_ / maxSimTime_ * 100. : double(itrs_) / double(maxIters_) * 100.;
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count();
    std::ostringstream m;
    m << "Simulation completion (%) |      " << pct << "\n"
      << "Iterations completed      |      " << itrs_ << "\n"
      << "Simulation time (sec)     |      " << simTime_ << "\n"
      << "Elapsed time (s)          |      " << secs << "\n"
      << "Residual norm             |      " << residualNorm;
    Output::print("RunControl", m.str());
    Output::printLine();
}

void RunControl::displayEndMessage() { Output::print("RunControl", "Simulation complete."); }

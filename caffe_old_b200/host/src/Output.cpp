// Console output and exceptions of the host layer.
#include "Output.h"

#include <iostream>

namespace {
thread_local std::string g_exceptionText;
}

void Output::print(const std::string& message) { std::cout << message << std::endl; }

void Output::print(const std::string& className, const std::string& message) { std::cout << className << ": " << message << std::endl; }

void Output::raiseException(std::string className, std::string methodName, std::string problemDescription) {
    g_exceptionText = "in \"" + className + "::" + methodName + "\", " + problemDescription;
    throw g_exceptionText.c_str();
}

void Output::issueWarning(std::string className, std::string methodName, std::string warningDescription) {
    std::cerr << "Warning in \"" << className << "::" << methodName << "\": " << warningDescription << std::endl;
}

void Output::printCaffeHeader() { print("CAFFE finite-volume solvers, B200 device library"); }

void Output::printLine() { std::cout << "------------------------------------------------------------" << std::endl; }

// Console output and error reporting of the host layer (reference: src/RunControl/Output.h).
// raiseException throws a const char* (the message stays valid until the next exception),
// which the module mains catch.
#pragma once
#include <string>

class Output {
public:
    static void print(const std::string& message);
    static void print(const std::string& className, const std::string& message);
    static void raiseException(std::string className, std::string methodName, std::string problemDescription);
    static void issueWarning(std::string className, std::string methodName, std::string warningDescription);
    static void printCaffeHeader();
    static void printLine();
};

// MGBrain C++ API: command-line parameters of the benchmark programs
// (src/util/parser.h:7-96): --name=value pairs with the reference's names
// and defaults (--nsyn=10000, --npart=1, --model=model, --file=tmp.txt,
// --prefix=../../benchdata/, --rate=0.002).
#pragma once
#include <sstream>
#include <string>
#include <unordered_map>

namespace MGBrain {

class ParamsParser {
    std::unordered_map<std::string, std::string> params;

public:
    static std::string NSYN, NPART, MODEL, FILE, PREFIX, RATE;
    ParamsParser(int args, char* argv[]);
    std::string getStr(std::string name);
    size_t getNum(std::string name);
    float getFloat(std::string name);
    bool getBool(std::string name);
};

}  // namespace MGBrain

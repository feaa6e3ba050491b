// host_util.h — input-file and forcing-file readers of the APT driver.
//
// Same semantics as the reference's helper.cpp: a parameter line is a
// whitespace-separated token stream in which `key = value` sets the parameter
// (getParam, 3DgrainMPI/helper.cpp:44-74; the int overload parses through stof
// and truncates); a forcing file holds one number per line (read_input,
// helper.cpp:77-101).  Unlike the reference, reads are bounded by the caller's
// capacity and report how many values were read.
#pragma once

#include <string>
#include <vector>

namespace cupf_host {

// Sets `param` from every `key = value` token triple on the line (last wins).
// Returns true if the key was found with an '=' and a value.
bool getParam(const std::string& lineText, const std::string& key, float& param);
bool getParam(const std::string& lineText, const std::string& key, int& param);

// Reads up to `cap` numbers, one per line (the first token of each line).
// Returns the number of lines read, or -1 if the file cannot be opened.
int read_input(const std::string& path, float* target, int cap);
int read_input(const std::string& path, int* target, int cap);
std::vector<float> read_column(const std::string& path);

}  // namespace cupf_host

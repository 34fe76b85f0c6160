/*
 * Process-grid parameters of the class-level API (the reference's command_line.h:19-27, command_line.cpp:31-84):
 * ReadParam reads "gridx = n" ... "gridt = n" lines from standard input.  kuqcd_init reads them only when
 * KUQCD_GRID_STDIN=1; the grid must be 1x1x1x1 (one GPU per process).  Unset entries default to 1.
 */
#ifndef COMMAND_LINE_H
#define COMMAND_LINE_H

#include <iostream>
#include <string>

namespace kuqcd {

/* s without leading and trailing blanks */
inline std::string Trim(const std::string &s)
{
    const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

class CmdLineParam {
public:
    int gridx = 1, gridy = 1, gridz = 1, gridt = 1;
    void ReadParam()
    {
        std::string line;
        while (std::getline(std::cin, line)) {
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            const std::string key = Trim(line.substr(0, eq));
            int *dst = key == "gridx" ? &gridx : key == "gridy" ? &gridy : key == "gridz" ? &gridz
                     : key == "gridt" ? &gridt : nullptr;
            if (!dst) continue;
            try {
                *dst = std::stoi(Trim(line.substr(eq + 1)));
            } catch (...) {
            }
        }
    }
};

}  // namespace kuqcd

#endif

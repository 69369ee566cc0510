// user_input.hpp -- the interactive prompts of the reference's programs
// (src/core/userinput.cpp), shared by match_template and refine_template.
#pragma once
#include <unistd.h>

#include <cctype>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "prep.hpp"

namespace tmhost {

// UserInput (src/core/userinput.cpp:40-110): question [default] padded to 50
// columns, " : ", one line from stdin; empty = default on a terminal and an
// error when scripted; '*' exits; '?' shows the help text and asks again.
class UserInput {
public:
    UserInput() : tty_(isatty(0)) {}
    std::string ask(const char* q, const char* help, const char* def) {
        for (;;) {
            std::string shown = std::string(q) + (def[0] && tty_ ? std::string(" [") + def + "]" : "");
            std::printf("%s", shown.c_str());
            for (int k = (int)shown.size(); k < 50; k++) std::printf(" ");
            std::printf(" : ");
            std::fflush(stdout);
            std::string line;
            if (!std::getline(std::cin, line)) {
                std::printf("\n Error: input ended before every question was answered, exiting...\n\n");
                std::exit(-1);
            }
            if (!line.empty() && line[0] == '*') std::exit(0);
            if (line.empty()) {
                if (!tty_) {
                    std::printf("\n Error: Blank answer in scripted mode, exiting...\n\n");
                    std::exit(-1);
                }
                line = def;
            } else if (line[0] == '?') {
                std::printf("\n%s\n\n", help);
                continue;
            }
            if (!tty_) std::printf("%s\n", line.c_str());
            return line;
        }
    }
    std::string filename(const char* q, const char* help, const char* def, bool must_exist) {
        for (;;) {
            std::string f = ask(q, help, def);
            if (!must_exist || access(f.c_str(), R_OK) == 0) return f;
            std::printf("\nError: File does not exist, please provide an existing file!\n\n");
            if (!tty_) std::exit(-1);
        }
    }
    float number(const char* q, const char* help, const char* def, float lo = -FLT_MAX, float hi = FLT_MAX) {
        for (;;) {
            std::string s = ask(q, help, def);
            char* end = nullptr;
            const float v = std::strtof(s.c_str(), &end);
            if (end != s.c_str() && v >= lo && v <= hi) return v;
            std::printf("\nError: Number outside of acceptable range!\n\n");
            if (!tty_) std::exit(-1);
        }
    }
    bool yes_no(const char* q, const char* help, const char* def) {
        for (;;) {
            std::string s = ask(q, help, def);
            if (s[0] == 'y' || s[0] == 'Y') return true;
            if (s[0] == 'n' || s[0] == 'N') return false;
            std::printf("\n Error: answer is not recognized...\n\n");
            if (!tty_) std::exit(-1);
        }
    }
    std::string symmetry(const char* q, const char* help, const char* def) {
        for (;;) {
            std::string s = ask(q, help, def);
            for (auto& c : s) c = (char)toupper(c);
            if (!search_grid(15.0f, s).empty()) return s;
            std::printf("\nError: Unrecognized symmetry!\n\n");
            if (!tty_) std::exit(-1);
        }
    }

private:
    bool tty_;
};

}  // namespace tmhost

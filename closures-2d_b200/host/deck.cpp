// deck.cpp -- see deck.h (input_deck_reader.cpp:17-171).
#include "deck.h"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace clb {

static std::string lower(const std::string &s)
{
    std::string r(s);
    for (auto &c : r)
        c = (char)std::tolower((unsigned char)c);
    return r;
}

bool InputDeck::read(const char *filename)
{
    FILE *f = std::fopen(filename, "r");
    if (!f) {
        std::printf("Could not open file.\n");
        return false;
    }
    char line[500];
    int lineNumber = 0;
    KV kv;
    while (std::fgets(line, sizeof(line), f)) {
        lineNumber++;
        if (char *nl = std::strchr(line, '\n'))
            *nl = 0;
        if (char *c = std::strchr(line, '#'))
            *c = 0;
        char *save = nullptr;
        char *tok = strtok_r(line, " \t", &save);
        if (!tok)
            continue;
        kv.key.assign(tok, strnlen(tok, VALUE_CHAR_LEN - 1));
        tok = strtok_r(nullptr, " ", &save);
        if (tok)
            kv.value.assign(tok, strnlen(tok, VALUE_CHAR_LEN - 1));
        else
            std::printf("Error in input file at line: %d\n", lineNumber);
        tok = strtok_r(nullptr, " ", &save);
        if (!tok)
            kv_.push_back(kv);
        else
            std::printf("Error in input file at line: %d\n", lineNumber);
    }
    std::fclose(f);
    return true;
}

bool InputDeck::get(const char *key, std::string &value) const
{
    std::string k = lower(key);
    for (const auto &e : kv_) {
        if (lower(e.key) == k) {
            value = lower(e.value);
            return true;
        }
    }
    return false;
}

bool InputDeck::get(const char *key, int *value) const
{
    std::string s;
    if (!get(key, s))
        return false;
    *value = std::atoi(s.c_str());
    return true;
}

bool InputDeck::get(const char *key, double *value) const
{
    std::string s;
    if (!get(key, s))
        return false;
    *value = std::atof(s.c_str());
    return true;
}

void InputDeck::print() const
{
    std::printf("--- Input Deck ---\n");
    for (const auto &e : kv_)
        std::printf("%s = %s\n", e.key.c_str(), e.value.c_str());
}

}  // namespace clb

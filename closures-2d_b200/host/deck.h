// deck.h -- input.deck reader with the reference's semantics
// (src/input_deck_reader.{h,cpp}): '#' comments, first token the key, second
// the value, lines with a third token rejected, keys matched
// case-insensitively, values lowercased, atoi/atof conversion.
#pragma once
#include <string>
#include <vector>

namespace clb {

class InputDeck {
public:
    static const int VALUE_CHAR_LEN = 128;
    // Returns false if the file cannot be opened (the reference prints
    // "Could not open file." and continues with an empty deck).
    bool read(const char *filename);
    bool get(const char *key, std::string &value) const;
    bool get(const char *key, int *value) const;
    bool get(const char *key, double *value) const;
    void print() const;

private:
    struct KV {
        std::string key, value;
    };
    std::vector<KV> kv_;
};

}  // namespace clb

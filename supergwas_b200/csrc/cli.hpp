// cli.hpp -- the command-line grammar shared by the kgwas and kgwas_2d
// programs.
//
// Both take a fixed number of leading words, then a tail read left to right:
// "--name VALUE" options (a name with no word after it is not an option) and
// other words.  What differs between them -- which options exist, whether the
// first tail word may be a positional threshold, what an unknown word means
// -- is data in a Grammar, so each program states its command line as a
// table (src/kgwas.cpp:67-126, src/kgwas_2d.cpp:44-76).
#pragma once
#include <cstdlib>
#include <functional>
#include <string>
#include <vector>

namespace kgcli {

struct Option {
  const char* name;
  std::function<void(const std::string&)> take;  // receives the next word
};

struct Grammar {
  int required = 0;                               // leading words
  std::function<void(const char* prog)> usage;    // too few words: print it, exit(1)
  // A first tail word that `leading_accept` admits is a positional value,
  // handed to `leading_take` before the options are read.
  std::function<bool(const std::string&)> leading_accept;
  std::function<void(const std::string&)> leading_take;
  std::vector<Option> options;
  std::function<void(const std::string&)> other;  // any other tail word; unset: ignored
};

// Returns the required leading words.
inline std::vector<std::string> parse(int argc, char** argv, const Grammar& g) {
  if (argc - 1 < g.required) {
    g.usage(argv[0]);
    std::exit(1);
  }
  std::vector<std::string> lead(argv + 1, argv + 1 + g.required);
  int i = 1 + g.required;
  if (g.leading_accept && i < argc && g.leading_accept(argv[i])) g.leading_take(argv[i++]);
  while (i < argc) {
    const std::string word = argv[i];
    const Option* hit = nullptr;
    if (i + 1 < argc)
      for (const Option& o : g.options)
        if (word == o.name) {
          hit = &o;
          break;
        }
    if (hit) {
      hit->take(argv[i + 1]);
      i += 2;
    } else {
      if (g.other) g.other(word);
      ++i;
    }
  }
  return lead;
}

}  // namespace kgcli

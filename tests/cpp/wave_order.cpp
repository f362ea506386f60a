// Reads graphs from stdin, one per line: N, then N forward flags, then N successors (a successor
// >= N is no edge); prints the wave order graphflow::devflow::waveOrder gives, one line each.
#include <cstdint>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "wave_order.hpp"

int main()
{
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::uint32_t n = 0;
        if (!(in >> n))
            continue;
        std::vector<char> forwards(n, 0);
        std::vector<std::uint32_t> succ(n, 0u);
        for (auto& f : forwards) {
            int v = 0;
            in >> v;
            f = static_cast<char>(v);
        }
        for (auto& s : succ)
            in >> s;
        const auto seq = graphflow::devflow::waveOrder(forwards, succ);
        for (std::size_t i = 0; i < seq.size(); ++i)
            std::cout << (i ? " " : "") << seq[i];
        std::cout << "\n";
    }
    return 0;
}

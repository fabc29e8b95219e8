// Test stand-in for the AudioFile library (an empty submodule in the
// Snipet/VIRS tree): the members that VectorSpace and the dispatch binding
// touch -- the per-channel sample buffers and the channel length.
#pragma once

#include <vector>

template <class T> class AudioFile {
public:
    std::vector<std::vector<T>> samples;
    int getNumSamplesPerChannel() const { return samples.empty() ? 0 : (int)samples[0].size(); }
};

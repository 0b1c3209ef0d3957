// hornets_nest::StaticAlgorithm (primitives/HornetAlg.cuh:51-150): the
// run / reset / release / validate interface every algorithm implements.
#pragma once

namespace hornets_nest {

template <typename HornetClass>
class StaticAlgorithm {
public:
    explicit StaticAlgorithm(HornetClass& hornet) noexcept : hornet(hornet) {}
    virtual ~StaticAlgorithm() noexcept = default;
    virtual void run() = 0;
    virtual void reset() = 0;
    virtual void release() = 0;
    virtual bool validate() = 0;

    using VertexType = typename HornetClass::VertexType;
    using DegreeType = typename HornetClass::DegreeType;

protected:
    HornetClass& hornet;
};

}  // namespace hornets_nest

// Drop-in forwarding, assembly half: the apps' InitializeMassAndStiffness
// calls (MassAndStiffness.h:490-495) go to a wrapper that runs the reference's
// assembly and records the operator for the device system (gdtp_dropin.inl
// explains the whole layer).
#pragma once

#include "gdtp_dropin.inl"

namespace gdtp_dropin {

// InitializeMassAndStiffness (MassAndStiffness.h:490-495): the reference's
// assembly (its outputs feed the apps' right-hand sides and direct solver),
// and the metric recorded for the device assembly of this operator.
inline int InitializeMassAndStiffness(std::vector<double>& deepMassCoefficients, std::vector<double>& deepStiffnessCoefficients,
                                      SparseMatrix<double, int>& boundaryBoundaryMassMatrix,
                                      SparseMatrix<double, int>& boundaryBoundaryStiffnessMatrix,
                                      SparseMatrix<double, int>& boundaryDeepMassMatrix, SparseMatrix<double, int>& boundaryDeepStiffnessMatrix,
                                      const HierarchicalSystem& hierarchy,
                                      const std::vector<std::vector<SquareMatrix<double, 2>>>& parameterMetric,
                                      const std::vector<AtlasChart>& atlasCharts, const BoundaryProlongationData& boundaryProlongation,
                                      bool computeCellBasedStiffness, const std::vector<Point3D<double>>& inputSignal,
                                      std::vector<double>& texelToCellCoeffs, SparseMatrix<double, int> boundaryCellBasedStiffnessRHSMatrix[3]) {
  const int result = ::InitializeMassAndStiffness(deepMassCoefficients, deepStiffnessCoefficients, boundaryBoundaryMassMatrix,
                                                  boundaryBoundaryStiffnessMatrix, boundaryDeepMassMatrix, boundaryDeepStiffnessMatrix,
                                                  hierarchy, parameterMetric, atlasCharts, boundaryProlongation, computeCellBasedStiffness,
                                                  inputSignal, texelToCellCoeffs, boundaryCellBasedStiffnessRHSMatrix);
  if (!result) return result;
  OperatorRecord& op = operators()[&deepMassCoefficients];
  if (op.system) gdtp_system_free(op.system);
  op = OperatorRecord();
  op.hierarchy = &hierarchy;
  size_t nt = 0;
  for (const AtlasChart& c : atlasCharts)
    for (int t : c.meshTriangleIndices) nt = std::max(nt, size_t(t) + 1);
  op.metric.assign(4 * nt, 0.0);
  for (size_t c = 0; c < atlasCharts.size() && c < parameterMetric.size(); c++)
    for (size_t k = 0; k < atlasCharts[c].meshTriangleIndices.size() && k < parameterMetric[c].size(); k++) {
      const size_t t = size_t(atlasCharts[c].meshTriangleIndices[k]);
      const SquareMatrix<double, 2>& g = parameterMetric[c][k];
      op.metric[4 * t] = g(0, 0);
      op.metric[4 * t + 1] = g(0, 1);
      op.metric[4 * t + 2] = g(1, 0);
      op.metric[4 * t + 3] = g(1, 1);
    }
  deep_arrays()[&deepMassCoefficients] = std::make_pair(static_cast<const void*>(&deepMassCoefficients), 1);
  deep_arrays()[&deepStiffnessCoefficients] = std::make_pair(static_cast<const void*>(&deepMassCoefficients), 2);
  return result;
}
// the reference's per-chart InitializeMassAndStiffness (MassAndStiffness.h:407) unchanged
template <class... A>
inline int InitializeMassAndStiffness(const std::vector<std::vector<SquareMatrix<double, 2>>>& parameterMetric, A&&... a) {
  return ::InitializeMassAndStiffness(parameterMetric, std::forward<A>(a)...);
}

}  // namespace gdtp_dropin

#define InitializeMassAndStiffness gdtp_dropin::InitializeMassAndStiffness

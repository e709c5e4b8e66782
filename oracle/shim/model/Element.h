// Test-infrastructure shim replacing the reference's model/Element.h, whose
// only job beyond holding the element's node list is the element volume V_e,
// computed there with VTK (absent in this image).
//
// V_e here is the volume enclosed by the element's CORNER nodes, every face
// triangulated (quad a-b-c-d -> a-b-c + a-c-d), by the divergence theorem.
// For straight-edged elements with planar faces this equals the exact volume
// that VTK's triangulated-surface volume also returns; the CUDA path and the C
// restatement in oracle/efem_oracle.c use this same definition.
#pragma once
#include "Eigen/Dense"
#include "core/Object.h"
#include "model/Node.h"
#include <cmath>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

namespace EFEM {
class Element : public Object {
public:
    std::vector<int> node_indexs;
    std::vector<std::shared_ptr<Node>> nodes;
    int material_id;
    std::unordered_map<std::string, std::shared_ptr<Object>> extra_info;

    void init() { }

    double volume()
    {
        auto p = [this](int i) -> Eigen::Vector3d { return nodes[i]->position + nodes[i]->dx; };
        if (nodes.size() == 4 || nodes.size() == 10) {
            Eigen::Vector3d a = p(1) - p(0), b = p(2) - p(0), c = p(3) - p(0);
            return std::fabs(a.dot(b.cross(c))) / 6.0;
        }
        // hexahedron corners 0..7 in the usual two-loop order (both the
        // 8-node and the 20-node element number their corners this way)
        static const int faces[6][4] = { { 0, 3, 2, 1 }, { 4, 5, 6, 7 }, { 0, 1, 5, 4 },
            { 1, 2, 6, 5 }, { 2, 3, 7, 6 }, { 3, 0, 4, 7 } };
        double v6 = 0.0;
        for (int f = 0; f < 6; f++) {
            Eigen::Vector3d a = p(faces[f][0]), b = p(faces[f][1]), c = p(faces[f][2]), d = p(faces[f][3]);
            v6 += a.dot(b.cross(c)) + a.dot(c.cross(d));
        }
        return std::fabs(v6) / 6.0;
    }
};
}

/* Build shim: FlowLB's cudaUtils.cuh names FLB::Texture2D only in the
 * declaration of its OpenGL texture helper, which the solver path never calls. */
#pragma once
namespace FLB { class Texture2D; }

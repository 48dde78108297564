// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,12,1,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,12,1,12>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1920,120,12,10,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1920,120,12,10,16>(const PassDesc);
extern const StaticPlan kPlans_f64_3[];
extern const int kPlansCount_f64_3;
const StaticPlan kPlans_f64_3[] = {
  {4, 1, 1, {4}, 1024, (const void*)&axis_pass_static<double,true,1024,4,1,4>, (const void*)&axis_pass_static<double,false,1024,4,1,4>, nullptr, nullptr, 512},
  {12, 1, 1, {12}, 512, (const void*)&axis_pass_static<double,true,512,12,1,12>, (const void*)&axis_pass_static<double,false,512,12,1,12>, (const void*)&axis_pass_pipe<double,512,false,12,1,12>, (const void*)&axis_pass_pipe<double,512,true,12,1,12>, 512},
  {25, 5, 2, {5,5}, 1024, (const void*)&axis_pass_static<double,true,1024,25,5,5,5>, (const void*)&axis_pass_static<double,false,1024,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,false,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,true,25,5,5,5>, 512},
  {45, 3, 2, {15,3}, 512, (const void*)&axis_pass_static<double,true,512,45,3,15,3>, (const void*)&axis_pass_static<double,false,512,45,3,15,3>, (const void*)&axis_pass_pipe<double,512,false,45,3,15,3>, (const void*)&axis_pass_pipe<double,512,true,45,3,15,3>, 512},
  {72, 6, 2, {12,6}, 512, (const void*)&axis_pass_static<double,true,512,72,6,12,6>, (const void*)&axis_pass_static<double,false,512,72,6,12,6>, (const void*)&axis_pass_pipe<double,512,false,72,6,12,6>, (const void*)&axis_pass_pipe<double,512,true,72,6,12,6>, 512},
  {100, 10, 2, {10,10}, 512, (const void*)&axis_pass_static<double,true,512,100,10,10,10>, (const void*)&axis_pass_static<double,false,512,100,10,10,10>, (const void*)&axis_pass_pipe<double,512,false,100,10,10,10>, (const void*)&axis_pass_pipe<double,512,true,100,10,10,10>, 512},
  {144, 12, 2, {12,12}, 512, (const void*)&axis_pass_static<double,true,512,144,12,12,12>, (const void*)&axis_pass_static<double,false,512,144,12,12,12>, (const void*)&axis_pass_pipe<double,512,false,144,12,12,12>, (const void*)&axis_pass_pipe<double,512,true,144,12,12,12>, 512},
  {200, 25, 3, {5,5,8}, 512, (const void*)&axis_pass_static<double,true,512,200,25,5,5,8>, (const void*)&axis_pass_static<double,false,512,200,25,5,5,8>, (const void*)&axis_pass_pipe<double,512,false,200,25,5,5,8>, (const void*)&axis_pass_pipe<double,512,true,200,25,5,5,8>, 512},
  {256, 16, 2, {16,16}, 512, (const void*)&axis_pass_static<double,true,512,256,16,16,16>, (const void*)&axis_pass_static<double,false,512,256,16,16,16>, (const void*)&axis_pass_pipe<double,512,false,256,16,16,16>, (const void*)&axis_pass_pipe<double,512,true,256,16,16,16>, 512},
  {360, 36, 3, {10,6,6}, 512, (const void*)&axis_pass_static<double,true,512,360,36,10,6,6>, (const void*)&axis_pass_static<double,false,512,360,36,10,6,6>, (const void*)&axis_pass_pipe<double,512,false,360,36,10,6,6>, (const void*)&axis_pass_pipe<double,512,true,360,36,10,6,6>, 512},
  {450, 30, 3, {15,6,5}, 512, (const void*)&axis_pass_static<double,true,512,450,30,15,6,5>, (const void*)&axis_pass_static<double,false,512,450,30,15,6,5>, (const void*)&axis_pass_pipe<double,512,false,450,30,15,6,5>, (const void*)&axis_pass_pipe<double,512,true,450,30,15,6,5>, 512},
  {576, 48, 3, {12,6,8}, 512, (const void*)&axis_pass_static<double,true,512,576,48,12,6,8>, (const void*)&axis_pass_static<double,false,512,576,48,12,6,8>, nullptr, nullptr, 512},
  {720, 60, 3, {12,10,6}, 512, (const void*)&axis_pass_static<double,true,512,720,60,12,10,6>, (const void*)&axis_pass_static<double,false,512,720,60,12,10,6>, nullptr, nullptr, 512},
  {864, 72, 3, {12,12,6}, 512, (const void*)&axis_pass_static<double,true,512,864,72,12,12,6>, (const void*)&axis_pass_static<double,false,512,864,72,12,12,6>, nullptr, nullptr, 512},
  {1080, 72, 3, {15,12,6}, 512, (const void*)&axis_pass_static<double,true,512,1080,72,15,12,6>, (const void*)&axis_pass_static<double,false,512,1080,72,15,12,6>, nullptr, nullptr, 512},
  {1280, 80, 3, {10,16,8}, 512, (const void*)&axis_pass_static<double,true,512,1280,80,10,16,8>, (const void*)&axis_pass_static<double,false,512,1280,80,10,16,8>, nullptr, nullptr, 512},
  {1536, 96, 3, {12,16,8}, 512, (const void*)&axis_pass_static<double,true,512,1536,96,12,16,8>, (const void*)&axis_pass_static<double,false,512,1536,96,12,16,8>, nullptr, nullptr, 512},
  {1920, 120, 3, {12,10,16}, 512, (const void*)&axis_pass_static<double,true,512,1920,120,12,10,16>, (const void*)&axis_pass_static<double,false,512,1920,120,12,10,16>, nullptr, nullptr, 512},
};
const int kPlansCount_f64_3 = 18;
}  // namespace dfft

/*
 * Minimal stand-in for <vulkan/vulkan.h>, used ONLY to compile the
 * reference's GPU-free C sources (decoder, host encoder, CPU ME) into the
 * test oracle under oracle/_ref. The reference's gpu_compute.h names Vulkan
 * handle types in its context struct; nothing compiled here ever calls
 * Vulkan, so every handle is an opaque pointer and every enum a plain int.
 * This file is test infrastructure and is never part of the product library.
 */
#ifndef B200ENC_REF_VULKAN_STUB_H
#define B200ENC_REF_VULKAN_STUB_H
#include <stdint.h>
#define VK_NULL_HANDLE 0
#define VK_STUB_HANDLE(name) typedef struct name##_stub_T *name
VK_STUB_HANDLE(VkInstance);
VK_STUB_HANDLE(VkPhysicalDevice);
VK_STUB_HANDLE(VkDevice);
VK_STUB_HANDLE(VkQueue);
VK_STUB_HANDLE(VkCommandPool);
VK_STUB_HANDLE(VkCommandBuffer);
VK_STUB_HANDLE(VkDescriptorPool);
VK_STUB_HANDLE(VkDescriptorSetLayout);
VK_STUB_HANDLE(VkDescriptorSet);
VK_STUB_HANDLE(VkPipelineLayout);
VK_STUB_HANDLE(VkPipeline);
VK_STUB_HANDLE(VkBuffer);
VK_STUB_HANDLE(VkImage);
VK_STUB_HANDLE(VkImageView);
VK_STUB_HANDLE(VkDeviceMemory);
VK_STUB_HANDLE(VkFence);
VK_STUB_HANDLE(VkSemaphore);
VK_STUB_HANDLE(VkQueryPool);
VK_STUB_HANDLE(VkShaderModule);
typedef uint64_t VkDeviceSize;
typedef uint32_t VkFlags;
typedef int VkResult;
typedef int VkImageLayout;
typedef struct { uint32_t apiVersion; uint32_t vendorID; uint32_t deviceID; char deviceName[256]; float timestampPeriod; } VkPhysicalDeviceProperties;
typedef void *PFN_vkGetMemoryFdKHR;
typedef void *PFN_vkImportSemaphoreFdKHR;
typedef void *PFN_vkVoidFunction;
#define VK_IMAGE_LAYOUT_UNDEFINED 0
#define VK_IMAGE_LAYOUT_GENERAL 1
#define VK_IMAGE_LAYOUT_PREINITIALIZED 8
#define VK_MEMORY_PROPERTY_HOST_VISIBLE_BIT 0x2
#define VK_MEMORY_PROPERTY_HOST_COHERENT_BIT 0x4
#define VK_MEMORY_PROPERTY_HOST_CACHED_BIT 0x8
#define VK_SEMAPHORE_IMPORT_TEMPORARY_BIT 0x1
#define VK_SUCCESS 0
#endif

// Named-attribute payloads of the public API (flow/Attributes.hpp in the reference): a tag per
// attribute, Field<Tag, T>, Record<Fields...> with get<Tag>() / set<Tag>() / record[tag], Set<Tags...>
// of the attributes a node may touch, and RecordProxy, which restricts a record to such a set at
// compile time. A Record is a trivially copyable struct of its fields in declaration order; in
// SoAStorage every field is one device column.
//
//   GRAPHFLOW_TAG(Id, idTag);                        // struct IdTag, constexpr IdTag idTag
//   using IdField = graphflow::Field<IdTag, std::uint64_t>;
//   using Particle = graphflow::Record<IdField, WeightField>;
//   p[idTag] = 7; p.set<WeightTag>(1u);
#pragma once

#include <cstddef>
#include <cstdint>
#include <tuple>
#include <type_traits>
#include <utility>

#include "storage.cuh"

namespace graphflow {

// An attribute tag is an empty type derived from TagBase.
struct TagBase {
};

template <typename Tag, typename T>
struct Field {
    static_assert(std::is_base_of_v<TagBase, Tag> && std::is_empty_v<Tag>,
                  "graphflow::Field: the tag must be an empty type derived from graphflow::TagBase");
    static_assert(std::is_trivially_copyable_v<T>, "graphflow::Field: attribute values must be trivially copyable");
    using tag_type = Tag;
    using value_type = T;
};

template <typename... Tags>
struct Set {
    static constexpr std::size_t size = sizeof...(Tags);
    template <typename Tag>
    static constexpr bool contains = (std::is_same_v<Tag, Tags> || ...);
};

namespace detail {

template <typename Tag, typename... Tags>
constexpr std::size_t tagIndex()
{
    constexpr bool hits[] = {std::is_same_v<Tag, Tags>...};
    for (std::size_t i = 0; i < sizeof...(Tags); ++i)
        if (hits[i])
            return i;
    return sizeof...(Tags);
}

template <typename... Tags>
constexpr bool uniqueTags()
{
    if constexpr (sizeof...(Tags) == 0u) {
        return true;
    } else {
        constexpr std::size_t first[] = {tagIndex<Tags, Tags...>()...};
        for (std::size_t i = 0; i < sizeof...(Tags); ++i)
            if (first[i] != i)
                return false;
        return true;
    }
}

// One field's storage; the index keeps equal value types apart.
template <std::size_t I, typename F>
struct RecordLeaf {
    typename F::value_type value;
};

template <typename Seq, typename... Fields>
struct RecordBase;

template <std::size_t... I, typename... Fields>
struct RecordBase<std::index_sequence<I...>, Fields...> : RecordLeaf<I, Fields>... {
};

} // namespace detail

template <typename... Fields>
struct AttributeList {
    static_assert(sizeof...(Fields) > 0u, "graphflow: an attribute list holds at least one field");
    static_assert(detail::uniqueTags<typename Fields::tag_type...>(), "graphflow: attribute tags must be distinct");
    static constexpr std::size_t size = sizeof...(Fields);
    using attribute_set = Set<typename Fields::tag_type...>;
    template <typename Tag>
    static constexpr bool contains = (std::is_same_v<Tag, typename Fields::tag_type> || ...);
    template <typename Tag>
    static constexpr std::size_t index = detail::tagIndex<Tag, typename Fields::tag_type...>();
    template <typename Tag>
    using field_type = std::tuple_element_t<index<Tag>, std::tuple<Fields...>>;
    template <typename Tag>
    using value_type = typename field_type<Tag>::value_type;
};

template <typename... Fields>
using Attributes = AttributeList<Fields...>;

template <typename TAccess, typename TSet>
class RecordProxy;

namespace detail {
template <typename TRecord>
struct RefRecordAccess;
template <typename TRecord>
struct ConstRefRecordAccess;
} // namespace detail

template <typename... Fields>
class Record : private detail::RecordBase<std::index_sequence_for<Fields...>, Fields...> {
    using list = AttributeList<Fields...>;
    template <std::size_t I>
    using leaf = detail::RecordLeaf<I, std::tuple_element_t<I, std::tuple<Fields...>>>;

public:
    using attribute_list = list;
    using attribute_set = typename list::attribute_set;
    static constexpr std::size_t size = sizeof...(Fields);

    constexpr Record() = default;

    template <typename... Values>
        requires(sizeof...(Values) == sizeof...(Fields))
    __host__ __device__ constexpr explicit Record(Values&&... values)
    {
        assign(std::index_sequence_for<Fields...>{}, std::forward<Values>(values)...);
    }

    template <typename Tag>
    __host__ __device__ constexpr auto& get()
    {
        static_assert(list::template contains<Tag>, "graphflow::Record: get<Tag>() names an unknown attribute");
        return static_cast<leaf<list::template index<Tag>>&>(*this).value;
    }
    template <typename Tag>
    __host__ __device__ constexpr const auto& get() const
    {
        static_assert(list::template contains<Tag>, "graphflow::Record: get<Tag>() names an unknown attribute");
        return static_cast<const leaf<list::template index<Tag>>&>(*this).value;
    }
    template <typename Tag, typename U>
    __host__ __device__ constexpr void set(U&& value)
    {
        static_assert(list::template contains<Tag>, "graphflow::Record: set<Tag>() names an unknown attribute");
        static_cast<leaf<list::template index<Tag>>&>(*this).value = std::forward<U>(value);
    }
    template <typename Tag>
    __host__ __device__ constexpr auto& operator[](Tag)
    {
        return get<Tag>();
    }
    template <typename Tag>
    __host__ __device__ constexpr const auto& operator[](Tag) const
    {
        return get<Tag>();
    }
    // The I-th field in declaration order (storage columns).
    template <std::size_t I>
    __host__ __device__ constexpr auto& field()
    {
        return static_cast<leaf<I>&>(*this).value;
    }
    template <std::size_t I>
    __host__ __device__ constexpr const auto& field() const
    {
        return static_cast<const leaf<I>&>(*this).value;
    }

    // A view of this record restricted to the attributes of TSet.
    template <typename TSet = attribute_set>
    __host__ __device__ auto proxy() -> RecordProxy<detail::RefRecordAccess<Record>, TSet>;
    template <typename TSet = attribute_set>
    __host__ __device__ auto proxy() const -> RecordProxy<detail::ConstRefRecordAccess<Record>, TSet>;

private:
    template <std::size_t... I, typename... Values>
    __host__ __device__ constexpr void assign(std::index_sequence<I...>, Values&&... values)
    {
        ((static_cast<leaf<I>&>(*this).value = std::forward<Values>(values)), ...);
    }
};

namespace detail {

template <typename TRecord>
struct RefRecordAccess {
    using record_type = TRecord;
    TRecord* record = nullptr;
    template <typename Tag>
    __host__ __device__ constexpr auto& get() const
    {
        return record->template get<Tag>();
    }
    template <typename Tag, typename U>
    __host__ __device__ constexpr void set(U&& value) const
    {
        record->template set<Tag>(std::forward<U>(value));
    }
    __host__ __device__ constexpr TRecord load() const { return *record; }
    __host__ __device__ constexpr void store(const TRecord& value) const { *record = value; }
};

template <typename TRecord>
struct ConstRefRecordAccess {
    using record_type = TRecord;
    const TRecord* record = nullptr;
    template <typename Tag>
    __host__ __device__ constexpr const auto& get() const
    {
        return record->template get<Tag>();
    }
    __host__ __device__ constexpr TRecord load() const { return *record; }
};

template <typename TSet, typename TList>
struct SetCompatible;
template <typename... Tags, typename TList>
struct SetCompatible<Set<Tags...>, TList> : std::bool_constant<(TList::template contains<Tags> && ...)> {
};

} // namespace detail

// A record restricted to the attributes of TSet: get/set/operator[] outside the set do not compile.
template <typename TAccess, typename TSet>
class RecordProxy {
    static_assert(detail::SetCompatible<TSet, typename TAccess::record_type::attribute_list>::value,
                  "graphflow::RecordProxy: the set names a tag that is not an attribute of the record");

public:
    using access_type = TAccess;
    using set_type = TSet;
    using record_type = typename TAccess::record_type;

    constexpr RecordProxy() = default;
    __host__ __device__ constexpr explicit RecordProxy(access_type access) : m_access(access) {}

    template <typename Tag>
    __host__ __device__ constexpr decltype(auto) get() const
    {
        static_assert(TSet::template contains<Tag>, "graphflow::RecordProxy: get<Tag>() is outside the node's set");
        return m_access.template get<Tag>();
    }
    template <typename Tag, typename U>
    __host__ __device__ constexpr void set(U&& value)
    {
        static_assert(TSet::template contains<Tag>, "graphflow::RecordProxy: set<Tag>() is outside the node's set");
        m_access.template set<Tag>(std::forward<U>(value));
    }
    template <typename Tag>
    __host__ __device__ constexpr decltype(auto) operator[](Tag) const
    {
        return get<Tag>();
    }
    __host__ __device__ constexpr record_type load() const { return m_access.load(); }
    __host__ __device__ constexpr void store(const record_type& r) { m_access.store(r); }
    __host__ __device__ constexpr operator record_type() const { return load(); }

private:
    access_type m_access{};
};

template <typename TRecord, typename TSet>
using MutableRecordProxy = RecordProxy<detail::RefRecordAccess<TRecord>, TSet>;
template <typename TRecord, typename TSet>
using ConstRecordProxy = RecordProxy<detail::ConstRefRecordAccess<TRecord>, TSet>;

template <typename... Fields>
template <typename TSet>
__host__ __device__ auto Record<Fields...>::proxy() -> RecordProxy<detail::RefRecordAccess<Record>, TSet>
{
    return RecordProxy<detail::RefRecordAccess<Record>, TSet>{detail::RefRecordAccess<Record>{this}};
}
template <typename... Fields>
template <typename TSet>
__host__ __device__ auto Record<Fields...>::proxy() const -> RecordProxy<detail::ConstRefRecordAccess<Record>, TSet>
{
    return RecordProxy<detail::ConstRefRecordAccess<Record>, TSet>{detail::ConstRefRecordAccess<Record>{this}};
}

template <typename T>
inline constexpr bool isRecord = false;
template <typename... Fields>
inline constexpr bool isRecord<Record<Fields...>> = true;

// Every field of a record is one SoAStorage column, in declaration order.
template <typename... Fields>
struct SoAFields<Record<Fields...>> {
    static constexpr std::size_t count = sizeof...(Fields);
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        each(p, f, std::index_sequence_for<Fields...>{});
    }

private:
    template <typename P, typename F, std::size_t... I>
    __host__ __device__ static void each(P& p, F& f, std::index_sequence<I...>)
    {
        (f(p.template field<I>()), ...);
    }
};

} // namespace graphflow

// GRAPHFLOW_ATTRIBUTE(Id, std::uint64_t): struct IdTag and the alias IdField = Field<IdTag, T>.
#define GRAPHFLOW_ATTRIBUTE(Name, T)                                                                                   \
    struct Name##Tag : ::graphflow::TagBase {                                                                          \
    };                                                                                                                 \
    using Name##Field = ::graphflow::Field<Name##Tag, T>

// GRAPHFLOW_TAG(Id, idTag): struct IdTag and `inline constexpr IdTag idTag{}`, so record[idTag]
// reads or writes the attribute; GRAPHFLOW_TAG(Id) names the value IdTag_v.
#define GRAPHFLOW_TAG_ONE(Name)                                                                                        \
    struct Name##Tag : ::graphflow::TagBase {                                                                          \
    };                                                                                                                 \
    inline constexpr Name##Tag Name##Tag##_v {}
#define GRAPHFLOW_TAG_NAMED(Name, Variable)                                                                            \
    struct Name##Tag : ::graphflow::TagBase {                                                                          \
    };                                                                                                                 \
    inline constexpr Name##Tag Variable {}
#define GRAPHFLOW_TAG_SELECT(_1, _2, Macro, ...) Macro
#define GRAPHFLOW_TAG(...) GRAPHFLOW_TAG_SELECT(__VA_ARGS__, GRAPHFLOW_TAG_NAMED, GRAPHFLOW_TAG_ONE)(__VA_ARGS__)
